"""The HEVE short step (ATMOS_DYN_Tstep_short_fvm_heve,
scale_atmos_dyn_tstep_short_fvm_heve.F90:109-1518, without the momentum/theta
FCT branches) against the oracle's restatement, bit for bit: one stage for
every flux scheme, and the RK4 short step with HEVE registered as the short
step (ATMOS_DYN_Tstep_short_regist)."""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
SCHEMES = ["UD3", "CD4", "UD3KOREN1993", "CD2", "UD5", "CD6"]


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()


def _stage_kw(a, o, **over):
    kw = dict(a)
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    kw.update(over)
    return kw


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("stretched", [False, True])
@pytest.mark.parametrize("full", [False, True])
def test_heve_stage_bit_exact(lib, scheme, stretched, full):
    g = helpers.small_grid(IMAX=13, JMAX=9, KMAX=17, stretched=stretched, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, dtrk=0.5, full=full)
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short_heve(g, scheme, o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_short_fvm_heve(**_stage_kw(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), f"{n}: max rel diff {helpers.max_rel(o_gpu[n], o_ref[n]):.3e}"


def test_heve_device_entry_matches_host_entry(lib):
    import torch

    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20)
    c = helpers.small_case(g, "CD4")
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    o_host = helpers.stage_outputs(g, 0.0)
    lib.setup(g.index_dict(), "CD4", "CD4")
    lib.ATMOS_DYN_Tstep_short_fvm_heve(**_stage_kw(a, o_host))

    def dev(x):
        return torch.from_numpy(np.ravel(x, order="K").copy()).cuda() if isinstance(x, np.ndarray) and x.ndim >= 2 else x

    ad = {k: dev(v) for k, v in a.items()}
    od = {k: torch.zeros(v.size, dtype=torch.float64, device="cuda") for k, v in o_host.items()}
    lib.ATMOS_DYN_Tstep_short_fvm_heve_dev(**_stage_kw(ad, od))
    lib.check()
    for n, v in o_host.items():
        got = od[n].cpu().numpy().reshape(v.shape, order="F")
        assert np.array_equal(got, v), n


@pytest.mark.parametrize("scheme", ["UD3", "CD4", "UD5"])
def test_heve_rk4_bit_exact(lib, scheme):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    xs = {n: c.state[n].copy(order="F") for n in STATE}
    xs["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xs["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk4(g, scheme, xs, dict(a, dt=0.5), short="HEVE")
    lib.setup(g.index_dict(), scheme, scheme)
    lib.short_type("HEVE")
    kw = dict(a, **xg)
    kw.update(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
              BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=0.5)
    lib.ATMOS_DYN_Tinteg_short_rk4(**kw)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


def test_heve_ensemble_matches_members_alone():
    from scale_b200.ensemble import STATE as ESTATE, Ensemble

    cases = mkinit.ensemble(sizes=[(16, 12, 20), (8, 10, 16), (33, 17, 12)])

    def run(cs):
        e = Ensemble(cs)
        try:
            hevi.short_type("HEVE")
            e.run(4)
            return e.members()
        finally:
            e.close()

    together = run(cases)
    for m, c in enumerate(cases):
        alone = run([c])[0]
        for n in ESTATE:
            assert np.array_equal(together[m][n], alone[n]), f"member {m} {n}"


def test_heve_momentum_fct_is_refused(lib):
    g = helpers.small_grid()
    c = helpers.small_case(g)
    a = helpers.short_inputs(c, full=False)
    lib.setup(g.index_dict(), "UD3", "UD3")
    with pytest.raises(hevi.HeviError, match="FCT") as e:
        lib.ATMOS_DYN_Tstep_short_fvm_heve(**_stage_kw(a, helpers.stage_outputs(g), FLAG_FCT_MOMENTUM=True))
    assert e.value.code == 5
    with pytest.raises(hevi.HeviError, match="HEVI, HEVE"):
        lib.short_type("HIVI")
