"""The HEVI short step with terrain-following metrics: non-flat GSQRT, J13G,
J23G and map factors MAPF (scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089
with every metric term, and the flux routines' GSQRT/J13G/J23G/MAPF
arguments), against the oracle's restatement, bit for bit: one stage for
every flux scheme, the RK4 and RK3 short steps, the device entry against the
host entry; and the entries that take flat terrain only refuse it."""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
SCHEMES = ["UD3", "CD4", "UD3KOREN1993", "CD2", "UD5", "CD6"]
SHORT_KW = dict(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
                BND_W=False, BND_E=False, BND_S=False, BND_N=False)


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()


def with_terrain(a, g, seed=17, amp=0.05):
    """Seeded non-flat metrics: GSQRT and MAPF within amp of 1, J13G and J23G
    within amp of 0, at every point and staggering."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = dict(a)
    a["GSQRT"] = np.asfortranarray(1.0 + amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    a["J13G"] = np.asfortranarray(amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    a["J23G"] = np.asfortranarray(amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    a["MAPF"] = np.asfortranarray(1.0 + amp * rng.uniform(-1, 1, size=(g.IA, g.JA, 2, 4)))
    return a


def _stage_kw(a, o):
    kw = dict(a)
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    return kw


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("stretched", [False, True])
@pytest.mark.parametrize("full", [False, True])
def test_terrain_stage_bit_exact(lib, scheme, stretched, full):
    g = helpers.small_grid(IMAX=13, JMAX=9, KMAX=17, stretched=stretched, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = with_terrain(helpers.short_inputs(c, dtrk=0.5, full=full), g)
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short(g, scheme, o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_kw(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), f"{n}: max rel diff {helpers.max_rel(o_gpu[n], o_ref[n]):.3e}"


def test_terrain_device_entry_matches_host_entry(lib):
    import torch

    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20, stretched=True)
    c = helpers.small_case(g, "CD4")
    helpers.perturb_state(c)
    a = with_terrain(helpers.short_inputs(c, full=True), g)
    o_host = helpers.stage_outputs(g, 0.0)
    lib.setup(g.index_dict(), "CD4", "CD4")
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_kw(a, o_host))

    def dev(x):
        return torch.from_numpy(np.ravel(x, order="K").copy()).cuda() if isinstance(x, np.ndarray) and x.ndim >= 2 else x

    ad = {k: dev(v) for k, v in a.items()}
    od = {k: torch.zeros(v.size, dtype=torch.float64, device="cuda") for k, v in o_host.items()}
    lib.ATMOS_DYN_Tstep_short_fvm_hevi_dev(**_stage_kw(ad, od))
    lib.check()
    for n, v in o_host.items():
        got = od[n].cpu().numpy().reshape(v.shape, order="F")
        assert np.array_equal(got, v), n


def _short_inputs(g, scheme):
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = with_terrain(helpers.short_inputs(c, full=True), g)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    xs = {n: c.state[n].copy(order="F") for n in STATE}
    xs["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xs["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    return a, xs


@pytest.mark.parametrize("scheme", ["UD3", "CD4", "UD5"])
def test_terrain_rk4_bit_exact(lib, scheme):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True, halo=helpers.halo_of(scheme))
    a, xs = _short_inputs(g, scheme)
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk4(g, scheme, xs, dict(a, dt=0.5))
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tinteg_short_rk4(**a, **xg, **SHORT_KW, dt=0.5)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("tinteg", ["RK3", "RK3WS2002"])
def test_terrain_rk3_bit_exact(lib, tinteg):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True)
    a, xs = _short_inputs(g, "CD4")
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk3(g, "CD4", xs, dict(a, dt=0.5), ws2002=tinteg == "RK3WS2002")
    lib.setup(g.index_dict(), "CD4", "CD4")
    lib.tinteg_short_type(tinteg)
    lib.ATMOS_DYN_Tinteg_short_rk3(**a, **xg, **SHORT_KW, dt=0.5)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("full", [False, True])
def test_terrain_heve_stage_bit_exact(lib, scheme, full):
    g = helpers.small_grid(IMAX=13, JMAX=9, KMAX=17, stretched=True, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = with_terrain(helpers.short_inputs(c, dtrk=0.5, full=full), g)
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short_heve(g, scheme, o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_short_fvm_heve(**_stage_kw(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), f"{n}: max rel diff {helpers.max_rel(o_gpu[n], o_ref[n]):.3e}"


@pytest.mark.parametrize("scheme", ["CD4", "UD5"])
def test_terrain_heve_rk4_bit_exact(lib, scheme):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True, halo=helpers.halo_of(scheme))
    a, xs = _short_inputs(g, scheme)
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk4(g, scheme, xs, dict(a, dt=0.1), short="HEVE")
    lib.setup(g.index_dict(), scheme, scheme)
    lib.short_type("HEVE")
    lib.ATMOS_DYN_Tinteg_short_rk4(**a, **xg, **SHORT_KW, dt=0.1)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("scheme", ["UD3", "UD3KOREN1993", "UD5"])
@pytest.mark.parametrize("fct,along", [(False, True), (True, True), (True, False)])
def test_terrain_tracer_step_bit_exact(lib, scheme, fct, along):
    """ATMOS_DYN_Tstep_tracer_fvm_heve with GSQRT and the (IA,JA,2) MAPF slice
    (tstep_tracer_fvm_heve.F90:72-240 and the limiter's metric factors,
    common.F90:2051-2120), with a non-zero tracer num_diff."""
    from test_gpu_parity import _tracer_inputs

    g = helpers.small_grid(IMAX=12, JMAX=14, KMAX=16, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, _, _ = _tracer_inputs(g, c)
    m = with_terrain(dict(), g, seed=23)
    GS, MAPF = m["GSQRT"], np.asfortranarray(m["MAPF"][..., 0])
    ndq = np.asfortranarray(1e-4 * np.random.Generator(np.random.PCG64(3)).standard_normal(g.shape + (3,)))
    ref = np.full(g.shape, np.nan, order="F")
    oracle.tstep_tracer(g, scheme, ref, q, q0, rhoq, d0, d, mflx, ndq, GS, MAPF, 2.5, fct, along)
    got = np.full(g.shape, np.nan, order="F")
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_tracer_fvm_heve(QTRCo=got, QTRC=q, QTRC0=q0, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                        num_diff=ndq, GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ,
                                        RCDX=g.RCDX, RCDY=g.RCDY, dtl=2.5, FLAG_FCT_TRACER=fct,
                                        FLAG_FCT_ALONG_STREAM=along)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


@pytest.mark.parametrize("fct", [False, True])
def test_terrain_tracer_rk3_bit_exact(lib, fct):
    from test_gpu_parity import _tracer_inputs

    g = helpers.small_grid(IMAX=10, JMAX=12, KMAX=18, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, _, _ = _tracer_inputs(g, c)
    m = with_terrain(dict(), g, seed=29)
    GS, MAPF = m["GSQRT"], np.asfortranarray(m["MAPF"][..., 0])
    ref = q0.copy(order="F")
    oracle.tinteg_tracer_rk3(g, "UD3KOREN1993", ref, ref, rhoq, d0, d, mflx, g.zeros(3), GS, MAPF, 5.0, fct, True)
    got = q0.copy(order="F")
    lib.setup(g.index_dict(), "UD3", "UD3KOREN1993")
    lib.ATMOS_DYN_Tinteg_tracer_rk3(QTRC=got, QTRC0=got, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                    num_diff=g.zeros(3), GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ, RCDX=g.RCDX,
                                    RCDY=g.RCDY, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dtl=5.0,
                                    FLAG_FCT_TRACER=fct, FLAG_FCT_ALONG_STREAM=True)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


def test_terrain_divergence_bit_exact(lib):
    """ATMOS_DYN_divergence (scale_atmos_dyn_common.F90:1437-1515) with its
    J13G/J23G/GSQRT/MAPF terms."""
    g = helpers.small_grid(IMAX=13, JMAX=11, KMAX=15, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    m = with_terrain(dict(), g, seed=31)
    ref = np.full(g.shape, np.nan, order="F")
    oracle.divergence(g, ref, c.state, m["GSQRT"], m["J13G"], m["J23G"], 1.0, m["MAPF"])
    got = np.full(g.shape, np.nan, order="F")
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_divergence(DDIV=got, MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"], MOMY=c.state["MOMY"],
                             GSQRT=m["GSQRT"], J13G=m["J13G"], J23G=m["J23G"], J33G=1.0, MAPF=m["MAPF"],
                             RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, FDZ=g.FDZ)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


def test_flat_only_entries_refuse_terrain(lib):
    import torch

    g = helpers.small_grid()
    c = helpers.small_case(g)
    a = with_terrain(helpers.short_inputs(c, full=False), g)
    lib.setup(g.index_dict(), "UD3", "UD3")
    dev = {k: (torch.from_numpy(np.ravel(v, order="K").copy()).cuda() if isinstance(v, np.ndarray) and v.ndim >= 2 else v)
           for k, v in a.items()}
    f32 = {k: dev[k].float() for k in ("num_diff", "DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t", "DDIV")}
    x = {n: dev[n].clone() for n in STATE}
    flx = {n: torch.zeros(3 * g.shape[0] * g.shape[1] * g.shape[2], dtype=torch.float32, device="cuda")
           for n in ("mflx_hi", "tflx_hi")}
    kw = {k: v for k, v in dev.items() if k not in f32 and k not in STATE and k not in
          ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "dtrk")}
    with pytest.raises(hevi.HeviError, match="not supported") as e:
        lib.ATMOS_DYN_Tinteg_short_rk4_mixed_dev(**kw, **f32, **x, **flx, **SHORT_KW, dt=0.5)
    assert e.value.code == 5
    # the flat-terrain stage still runs after the refusal
    a_flat = helpers.short_inputs(c, full=False)
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_kw(a_flat, helpers.stage_outputs(g)))


@pytest.mark.parametrize("case,divdmp", [("dry", 0.0), ("dry", 0.05), ("moist_fct", 0.0)])
def test_terrain_large_step_parity(lib, case, divdmp):
    """The device-resident large step with terrain: the general-metric short
    step, the metric divergence for divergence damping and the tracer step
    with GSQRT/MAPF, against the oracle's large step (the tolerance of the
    flat large-step tests: the moist RT2P goes through pow())."""
    from test_gpu_parity import _field_err, _run_large_both

    c = mkinit.config(1, scale=0.3) if case == "dry" else mkinit.config(2, scale=0.04)
    m = with_terrain(dict(), c.g, seed=5, amp=0.02)
    st_ref, st_gpu = _run_large_both(c, 2, lib, divdmp=divdmp, metrics=(m["GSQRT"], m["J13G"], m["J23G"], m["MAPF"]))
    for n in STATE:
        assert np.isfinite(st_gpu[n]).all(), n
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for iq in range(c.QA):
        err = _field_err(st_gpu["QTRC"][..., iq], st_ref["QTRC"][..., iq], c.g)
        assert err <= 1e-10, f"QTRC[{iq}]: {err:.3e}"
