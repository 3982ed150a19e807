"""The halo exchange hook of the library (scale_hevi_set_halo_exchange) with
the decomposition's exchange (scale_b200/decomp.py) on one GPU: a 1x1
decomposition, whose exchange is the periodic fill done by torch copies, must
give the results of the library's own periodic halo bit for bit, through the
RK4 short step, the large step, the FCT tracer limiter (R+/R- exchanged
between its kernels) and the filter at ND_ORDER > 1 (its work arrays
exchanged between the calc_diff4 applications)."""
import numpy as np
import pytest

import helpers
from scale_b200 import decomp, hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
SHORT_KW = dict(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
                BND_W=False, BND_E=False, BND_S=False, BND_N=False)


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()  # also clears the hook


def _attach(g):
    dec = decomp.Decomposition(g.IMAX, g.JMAX, 1, 1, 0, g.halo)
    decomp.attach(hevi, dec, g.KA)


@pytest.mark.parametrize("scheme", ["CD4", "UD5"])
def test_hook_rk4_matches_periodic_halo(lib, scheme):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    x0 = {n: c.state[n].copy(order="F") for n in STATE}
    x0["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    x0["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    res = []
    for hook in (False, True):
        x = {n: v.copy(order="F") for n, v in x0.items()}
        lib.setup(g.index_dict(), scheme, scheme)
        if hook:
            _attach(g)
        for _ in range(2):
            lib.ATMOS_DYN_Tinteg_short_rk4(**a, **x, **SHORT_KW, dt=0.5)
        res.append(x)
        lib.set_halo_exchange(None)
        lib.finalize()
    for n in x0:
        assert np.array_equal(res[0][n], res[1][n], equal_nan=True), n


def test_hook_large_step_matches_periodic_halo(lib):
    from test_gpu_parity import _large_inputs

    c = mkinit.config(1, scale=0.3)
    g = c.g
    tp, GS, J13, J23, MAPF = _large_inputs(c)
    cor = np.zeros((g.IA, g.JA), order="F")
    res = []
    for hook in (False, True):
        st = {n: v.copy(order="F") for n, v in c.state.items()}
        out = dict(mflx_hi=g.zeros(3), tflx_hi=g.zeros(3), num_diff=g.zeros(5, 3))
        lib.setup(g.index_dict(), c.scheme, c.scheme_tracer)
        if hook:
            _attach(g)
        for _ in range(2):
            lib.ATMOS_DYN_Tstep_large_fvm_heve(
                DENS=st["DENS"], MOMZ=st["MOMZ"], MOMX=st["MOMX"], MOMY=st["MOMY"], RHOT=st["RHOT"], QTRC=None, QA=0,
                **out, RHOQ_tp=None, CORIOLI=cor, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY,
                RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY, PHI=c.ref["PHI"],
                GSQRT=GS, J13G=J13, J23G=J23, J33G=1.0, MAPF=MAPF, AQ_R=None, AQ_CV=None, AQ_CP=None, AQ_MASS=None,
                REF_dens=c.ref["REF_dens"], REF_pott=c.ref["REF_pott"], REF_pres=c.ref["REF_pres"], ND_COEF=c.nd_coef,
                ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=True, wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0,
                FLAG_FCT_TRACER=False, FLAG_FCT_ALONG_STREAM=True, DTLS=c.dtl, DTSS=c.dt,
                **{k: v for k, v in tp.items() if k != "RHOQ_tp"})
        res.append({**st, **out})
        lib.set_halo_exchange(None)
        lib.finalize()
    for n in res[0]:
        assert np.array_equal(res[0][n], res[1][n], equal_nan=True), n


@pytest.mark.parametrize("order", [2, 3])
def test_hook_high_order_filter_matches_periodic_halo(lib, order):
    g = helpers.small_grid(IMAX=13, JMAX=11, KMAX=17, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    res = []
    for hook in (False, True):
        nd = np.full(g.shape + (5, 3), np.nan, order="F")
        lib.setup(g.index_dict(), "UD3", "UD3")
        if hook:
            _attach(g)
        lib.ATMOS_DYN_numfilter_coef(num_diff=nd, DENS=c.state["DENS"], MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"],
                                     MOMY=c.state["MOMY"], RHOT=c.state["RHOT"], CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY,
                                     FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5, REF_dens=c.ref["REF_dens"],
                                     REF_pott=c.ref["REF_pott"], ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7,
                                     ND_USE_RS=True)
        res.append(nd)
        lib.set_halo_exchange(None)
        lib.finalize()
    assert np.array_equal(res[0], res[1], equal_nan=True)


@pytest.mark.parametrize("along", [True, False])
def test_hook_fct_tracer_matches_periodic_halo(lib, along):
    from test_gpu_parity import _tracer_inputs

    g = helpers.small_grid(IMAX=14, JMAX=12, KMAX=16, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ndq = np.asfortranarray(1e-6 * np.random.default_rng(9).normal(size=g.shape + (3,)))
    res = []
    for hook in (False, True):
        qq = q.copy(order="F")
        lib.setup(g.index_dict(), "UD3", "UD3")
        if hook:
            _attach(g)
        lib.ATMOS_DYN_Tinteg_tracer_rk3(QTRC=qq, QTRC0=q0, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                        num_diff=ndq, GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ, RCDX=g.RCDX,
                                        RCDY=g.RCDY, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dtl=5.0,
                                        FLAG_FCT_TRACER=True, FLAG_FCT_ALONG_STREAM=along)
        res.append(qq)
        lib.set_halo_exchange(None)
        lib.finalize()
    assert np.array_equal(res[0], res[1], equal_nan=True)


def test_hook_mixed_precision_matches_periodic_halo(lib):
    """The mixed path's FP32 fields (num_diff) reach the hook with 4-byte
    elements; the result equals the library's own halo bit for bit."""
    from test_gpu_mixed import run_short_steps

    c = mkinit.config(1, scale=0.3)
    plain = run_short_steps(c, 3, mixed=True)
    hooked = run_short_steps(c, 3, mixed=True, hook=True)
    for n in STATE:
        assert np.array_equal(plain[n], hooked[n]), n
