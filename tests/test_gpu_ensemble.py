"""Uneven ensembles: members of different sizes advanced together (every
kernel launch covers all members, or the whole short step is one persistent
launch) give, member by member, the same state bit for bit as each member
advanced alone by the single-domain path, which the parity tests compare with
the oracle. Also across the stage kernel's tile shapes, with the step replayed
as a CUDA graph, and on the mixed-precision path. The persistent step's grid
barriers are bounded: a barrier made to wait for a CTA that does not exist
ends the launch with an error status, and the library stays usable."""
import numpy as np
import pytest

from scale_b200 import hevi, mkinit
from scale_b200.ensemble import STATE, Ensemble

pytestmark = pytest.mark.gpu

SIZES = [(16, 12, 20), (24, 20, 24), (8, 10, 16), (33, 17, 12)]
NSTEPS = 6


def _alone(cases, nsteps, mixed=False, tile_x=0):
    out = []
    for c in cases:
        e = Ensemble([c], mixed=mixed)
        try:
            hevi.stage_shape(tile_x, 0)
            e.run(nsteps)
            out.append(e.members()[0])
        finally:
            e.close()
    return out


def _together(cases, nsteps, mixed=False, tile_x=0, raster=0, graph=False, persistent=False):
    e = Ensemble(cases, mixed=mixed, persistent=persistent)
    try:
        hevi.stage_shape(tile_x, raster)
        if graph:
            e.capture(1)  # one eager step, then the recorded one
            e.run(nsteps - 1)
        else:
            e.run(nsteps)
        launches = hevi.kernel_launches()
        return e.members(), launches
    finally:
        e.close()


def _same(a, b):
    for m, (x, y) in enumerate(zip(a, b)):
        for n in STATE:
            assert np.array_equal(x[n], y[n]), f"member {m} {n}: max diff {np.max(np.abs(x[n] - y[n])):.3e}"


@pytest.fixture(scope="module")
def cases():
    return mkinit.ensemble(sizes=SIZES)


@pytest.fixture(scope="module")
def alone(cases):
    return _alone(cases, NSTEPS)


def test_ensemble_matches_members_alone(cases, alone):
    got, _ = _together(cases, NSTEPS)
    _same(got, alone)
    for st in got:
        assert all(np.isfinite(st[n]).all() for n in STATE)


@pytest.mark.parametrize("tile_x,raster", [(8, 4), (4, 1), (16, 64)])
def test_ensemble_tile_shapes_give_identical_results(cases, alone, tile_x, raster):
    got, _ = _together(cases, NSTEPS, tile_x=tile_x, raster=raster)
    _same(got, alone)


def test_ensemble_graph_replay(cases, alone):
    got, _ = _together(cases, NSTEPS, graph=True)
    _same(got, alone)


def test_ensemble_one_launch_per_kernel(cases):
    # the launch count of a step does not depend on the number of members; the
    # fused stage form on both sides (a single domain would otherwise take the
    # tiled stage, two kernels per stage)
    _, l4 = _together(cases, 2, tile_x=16)
    _, l1 = _together(cases[:1], 2, tile_x=16)
    assert l4 == l1


def test_ensemble_mixed_precision_matches_members_alone(cases):
    # the FP32 arithmetic compiles with FMA contraction, which each kernel form
    # applies to its own code; the members alone take the fused form, as the
    # ensemble does (the FP64 comparisons above cross the forms bit for bit)
    _same(_together(cases, 4, mixed=True)[0], _alone(cases, 4, mixed=True, tile_x=16))


def test_ensemble_rejects_single_domain_entries(cases):
    e = Ensemble(cases[:2])
    try:
        with pytest.raises(hevi.HeviError, match="ensemble"):
            hevi.ATMOS_DYN_Tinteg_short_rk4_dev(
                PROG=None, mflx_hi=e.mflx, tflx_hi=e.tflx, DPRES0=e.DPRES0, RT2P=e.RT2P, CORIOLI=e.CORIOLI,
                num_diff=e.num_diff, wdamp_coef=e.wdamp, divdmp_coef=0.1, DDIV=e.tend["DENS_t"],
                FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True, PHI=e.ref["PHI"],
                GSQRT=e.GSQRT, J13G=e.J0, J23G=e.J0, J33G=1.0, MAPF=e.MAPF, REF_dens=e.ref["REF_dens"],
                REF_rhot=e.REF_rhot, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=1.0, **e.X, **e.tend,
                **{k: e.grid[k] for k in ("CDZ", "FDZ", "FDX", "FDY", "RCDZ", "RCDX", "RCDY", "RFDZ", "RFDX",
                                          "RFDY")})
        with pytest.raises(hevi.HeviError, match="ensemble"):
            hevi.domain_sum_dev(e.X["DENS"], e.grid["CDZ"], e.grid["CDX"], e.grid["CDY"])
    finally:
        e.close()


def test_autotuned_shape_gives_identical_results(cases, alone):
    e = Ensemble(cases)
    try:
        hevi.stage_autotune(True)
        e.run(NSTEPS)
        got = e.members()
        rep = hevi.autotune_report()
        tx, r = hevi.stage_shape_get()
    finally:
        e.close()
    _same(got, alone)
    assert rep["path"] == "fp64" and len(rep["candidates"]) == 9
    assert [tx, r] == rep["chosen"][:2]
    assert min(c[2] for c in rep["candidates"]) == rep["chosen"][2]


@pytest.mark.parametrize("scheme", ["UD5", "CD6"])
def test_six_point_ensemble_matches_members_alone(scheme):
    # members on a lateral halo of 3, advanced together and alone
    cases = mkinit.ensemble(sizes=SIZES[:3], scheme=scheme)
    assert all(c.g.IS == 4 for c in cases)
    _same(_together(cases, 4)[0], _alone(cases, 4))


# ---- the whole short step as one persistent launch ----
def test_persistent_step_matches_members_alone(cases, alone):
    got, launches = _together(cases, NSTEPS, persistent=True)
    _same(got, alone)
    assert launches == NSTEPS  # one launch per short step


def test_persistent_step_graph_replay(cases, alone):
    got, _ = _together(cases, NSTEPS, graph=True, persistent=True)
    _same(got, alone)


def test_persistent_step_single_domain(cases, alone):
    got, launches = _together(cases[1:2], NSTEPS, persistent=True)
    _same(got, alone[1:2])
    assert launches == NSTEPS


@pytest.mark.parametrize("scheme", ["UD5", "CD6"])
def test_persistent_six_point(scheme):
    cases = mkinit.ensemble(sizes=SIZES[:3], scheme=scheme)
    _same(_together(cases, 4, persistent=True)[0], _alone(cases, 4))


def test_persistent_mixed_matches_members_alone(cases):
    got = _together(cases, 4, mixed=True, persistent=True)[0]
    want = _alone(cases, 4, mixed=True, tile_x=16)
    for m, (x, y) in enumerate(zip(got, want)):
        for n in STATE:
            scale = np.max(np.abs(y[n]))
            err = np.max(np.abs(x[n] - y[n])) / scale if scale else np.max(np.abs(x[n]))
            # the same FP32 kernels' code; FMA contraction may differ between the two compiled forms
            assert err <= 1e-6, f"member {m} {n}: {err:.3e}"


def test_persistent_barrier_wait_is_bounded(cases):
    # every barrier waits for one CTA more than the grid has: the first one
    # expires after 50 ms, the launch ends and the status reports it
    e = Ensemble(cases[:2], persistent=True)
    try:
        e.run(1)
        hevi.check()
        assert hevi.persistent_grid() > 0
        hevi.persistent_wait(0.05, extra_arrivals=1)
        e.run(1)
        with pytest.raises(hevi.HeviError, match="grid barrier") as err:
            hevi.check()
        assert err.value.code == 3
        # the limit back to its default and no extra arrival: the next step completes
        hevi.persistent_wait(2.0, extra_arrivals=0)
        e.run(1)
        hevi.check()
    finally:
        e.close()


def test_persistent_step_refuses_other_integrators(cases):
    e = Ensemble(cases[:2], persistent=True)
    try:
        hevi.tinteg_short_type("RK3")
        with pytest.raises(hevi.HeviError, match="RK4 of HEVI"):
            e.run(1)
    finally:
        e.close()
