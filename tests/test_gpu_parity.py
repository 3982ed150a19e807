"""Parity of the CUDA path with the CPU oracle, through the C-ABI.

Bit-exact cases: one HEVI stage, the RK4 short step, the numerical filter and
the tracer steps see identical inputs on both sides; the kernels keep the
reference's operation order without FMA contraction, so every output value
must be identical (NaN sentinels mark cells the reference leaves unwritten and
must stay unwritten). The multi-step large-step runs go through pow() in the
moist RT2P preparation, where the GPU and glibc may differ in the last bit, so
they are held to the tolerance of the specification (max relative error 1e-10).
"""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()


def _stage_call_args(a, o):
    kw = {k: v for k, v in a.items()}
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    return kw


SCHEMES = ["UD3", "CD4", "UD3KOREN1993", "CD2", "UD5", "CD6"]


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("stretched", [False, True])
@pytest.mark.parametrize("full", [False, True])
def test_stage_bit_exact(lib, scheme, stretched, full):
    g = helpers.small_grid(IMAX=13, JMAX=9, KMAX=17, stretched=stretched, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, dtrk=0.5, full=full)
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short(g, scheme, o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_call_args(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), f"{n}: max rel diff {helpers.max_rel(o_gpu[n], o_ref[n]):.3e}"


def test_stage_device_entry_matches_host_entry(lib):
    import torch

    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20)
    c = helpers.small_case(g, "UD3")
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    o_host = helpers.stage_outputs(g, 0.0)
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_call_args(a, o_host))

    def dev(x):
        return torch.from_numpy(np.ravel(x, order="K").copy()).cuda() if isinstance(x, np.ndarray) and x.ndim >= 2 else x

    ad = {k: dev(v) for k, v in a.items()}
    od = {k: torch.zeros(v.size, dtype=torch.float64, device="cuda") for k, v in o_host.items()}
    lib.ATMOS_DYN_Tstep_short_fvm_hevi_dev(**_stage_call_args(ad, od))
    lib.check()
    for n, v in o_host.items():
        got = od[n].cpu().numpy().reshape(v.shape, order="F")
        assert np.array_equal(got, v), n


@pytest.mark.parametrize("scheme", SCHEMES)
def test_rk4_short_step_bit_exact(lib, scheme):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=scheme in ("CD4", "UD5"), halo=helpers.halo_of(scheme))
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    xs = {n: c.state[n].copy(order="F") for n in STATE}
    xs["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xs["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk4(g, scheme, xs, dict(a, dt=1.0))
    lib.setup(g.index_dict(), scheme, scheme)
    kw = dict(a, **xg)
    kw.update(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
              BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=1.0)
    lib.ATMOS_DYN_Tinteg_short_rk4(**kw)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("order,halo", [(1, 2), (2, 2), (3, 2), (1, 3), (2, 3)])
@pytest.mark.parametrize("stretched", [False, True])
def test_numfilter_bit_exact(lib, stretched, order, halo):
    g = helpers.small_grid(IMAX=15, JMAX=10, KMAX=19, stretched=stretched, halo=halo)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    ref_nd = g.zeros(5, 3)
    oracle.numfilter(g, ref_nd, c.state, c.ref, DT=0.5, ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7)
    got = np.full(g.shape + (5, 3), np.nan, order="F")
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_numfilter_coef(num_diff=got, DENS=c.state["DENS"], MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"],
                                 MOMY=c.state["MOMY"], RHOT=c.state["RHOT"], CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY,
                                 FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5, REF_dens=c.ref["REF_dens"],
                                 REF_pott=c.ref["REF_pott"], ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7,
                                 ND_USE_RS=True)
    for v in range(5):
        for d in range(3):
            assert helpers.same(got[..., v, d], ref_nd[..., v, d]), f"num_diff(:,:,:,{v+1},{d+1})"


@pytest.mark.parametrize("kmax,halo", [(20, 2), (36, 2), (64, 3), (96, 2)])
def test_numfilter_tiled_form_bit_exact(lib, kmax, halo):
    """The filter's tiled form (num_diff from tiles staged by bulk tensor
    copies; KA a multiple of 4 admits the tensor maps) against the column form
    and the oracle, bit for bit, with ragged tiles and chunks."""
    g = helpers.small_grid(IMAX=13, JMAX=10, KMAX=kmax, stretched=True, halo=halo)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    ref_nd = g.zeros(5, 3)
    oracle.numfilter(g, ref_nd, c.state, c.ref, DT=0.5, ND_COEF=1e-3, ND_ORDER=1, ND_SFC_FACT=0.7)
    res = []
    for tiled in (True, False):
        got = np.full(g.shape + (5, 3), np.nan, order="F")
        lib.setup(g.index_dict(), "UD3", "UD3")
        lib.numfilter_form(tiled)
        lib.ATMOS_DYN_numfilter_coef(num_diff=got, DENS=c.state["DENS"], MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"],
                                     MOMY=c.state["MOMY"], RHOT=c.state["RHOT"], CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY,
                                     FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5, REF_dens=c.ref["REF_dens"],
                                     REF_pott=c.ref["REF_pott"], ND_COEF=1e-3, ND_ORDER=1, ND_SFC_FACT=0.7,
                                     ND_USE_RS=True)
        lib.finalize()
        res.append(got)
    assert np.array_equal(res[0], res[1], equal_nan=True)
    for v in range(5):
        for d in range(3):
            assert helpers.same(res[0][..., v, d], ref_nd[..., v, d]), f"num_diff(:,:,:,{v+1},{d+1})"


def _tracer_inputs(g, c, seed=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    q0 = np.asfortranarray(np.clip(1e-3 + 5e-4 * rng.normal(size=g.shape), 0.0, None))
    mkinit.periodic_fill(q0, g)
    q = np.asfortranarray(q0 + 1e-5 * rng.normal(size=g.shape))
    mkinit.periodic_fill(q, g)
    dens0 = c.state["DENS"].copy(order="F")
    dens = np.asfortranarray(dens0 * (1.0 + 1e-4 * rng.normal(size=g.shape)))
    mkinit.periodic_fill(dens, g)
    mflx = np.asfortranarray(np.stack([c.state["MOMZ"], c.state["MOMX"], c.state["MOMY"]], axis=-1)
                             + 0.3 * rng.normal(size=g.shape + (3,)))
    mflx[: g.KS - 1, :, :, 0] = 0.0
    mflx[g.KE - 1 :, :, :, 0] = 0.0
    for n in range(3):
        mkinit.periodic_fill(mflx[..., n], g)
    rhoq = np.asfortranarray(1e-8 * rng.normal(size=g.shape))
    GS, _, _, MAPF = oracle.flat_metrics(g)
    return q0, q, dens0, dens, mflx, rhoq, GS, np.asfortranarray(MAPF[..., 0])


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("fct,along", [(False, True), (True, True), (True, False)])
def test_tracer_step_bit_exact(lib, scheme, fct, along):
    g = helpers.small_grid(IMAX=12, JMAX=14, KMAX=16, halo=helpers.halo_of(scheme))
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ref = np.full(g.shape, np.nan, order="F")
    oracle.tstep_tracer(g, scheme, ref, q, q0, rhoq, d0, d, mflx, g.zeros(3), GS, MAPF, 2.5, fct, along)
    got = np.full(g.shape, np.nan, order="F")
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_tracer_fvm_heve(QTRCo=got, QTRC=q, QTRC0=q0, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                        num_diff=g.zeros(3), GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ,
                                        RCDX=g.RCDX, RCDY=g.RCDY, dtl=2.5, FLAG_FCT_TRACER=fct,
                                        FLAG_FCT_ALONG_STREAM=along)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


@pytest.mark.parametrize("scheme", ["UD3", "CD6"])
@pytest.mark.parametrize("along", [True, False])
@pytest.mark.parametrize("kmax", [40, 17])
def test_tracer_fct_forms_bit_exact(lib, scheme, along, kmax):
    """The fused limiter (strips of 16 rows, tiles of 8 columns x 32 levels)
    and the three-kernel form on a domain that fills neither: 13 x 37 columns,
    40 levels (a second chunk of 8) or 17 (odd KA: no tensor map, so both
    settings run the three-kernel form)."""
    g = helpers.small_grid(IMAX=13, JMAX=37, KMAX=kmax, halo=helpers.halo_of(scheme), stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ref = np.full(g.shape, np.nan, order="F")
    oracle.tstep_tracer(g, scheme, ref, q, q0, rhoq, d0, d, mflx, g.zeros(3), GS, MAPF, 2.5, True, along)
    res = []
    for fused in (True, False):
        got = np.full(g.shape, np.nan, order="F")
        lib.setup(g.index_dict(), scheme, scheme)
        lib.tracer_fct_form(fused)
        lib.ATMOS_DYN_Tstep_tracer_fvm_heve(QTRCo=got, QTRC=q, QTRC0=q0, RHOQ_t=rhoq, DENS0=d0, DENS=d,
                                            mflx_hi=mflx, num_diff=g.zeros(3), GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ,
                                            RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, dtl=2.5, FLAG_FCT_TRACER=True,
                                            FLAG_FCT_ALONG_STREAM=along)
        lib.check()
        lib.finalize()
        res.append(got)
        assert helpers.same(got, ref), f"fused={fused}: max rel diff {helpers.max_rel(got, ref):.3e}"
    assert np.array_equal(res[0], res[1], equal_nan=True)


@pytest.mark.parametrize("tscheme", ["UD3", "UD3KOREN1993"])
@pytest.mark.parametrize("fct", [False, True])
def test_tracer_rk3_bit_exact(lib, fct, tscheme):
    g = helpers.small_grid(IMAX=10, JMAX=12, KMAX=18, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ref = q0.copy(order="F")
    oracle.tinteg_tracer_rk3(g, tscheme, ref, ref, rhoq, d0, d, mflx, g.zeros(3), GS, MAPF, 5.0, fct, True)
    got = q0.copy(order="F")
    lib.setup(g.index_dict(), "UD3", tscheme)
    lib.ATMOS_DYN_Tinteg_tracer_rk3(QTRC=got, QTRC0=got, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                    num_diff=g.zeros(3), GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ, RCDX=g.RCDX,
                                    RCDY=g.RCDY, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dtl=5.0,
                                    FLAG_FCT_TRACER=fct, FLAG_FCT_ALONG_STREAM=True)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


def _large_inputs(c):
    g = c.g
    tp = {n: g.zeros() for n in ("DENS_tp", "MOMZ_tp", "MOMX_tp", "MOMY_tp", "RHOT_tp")}
    if c.QA:
        tp["RHOQ_tp"] = g.zeros(c.QA)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    return tp, GS, J13, J23, MAPF


def _run_large_both(c, nlarge, lib, divdmp=0.0, nd_order=1, short="HEVI", tinteg="RK4", metrics=None):
    g = c.g
    tp, GS, J13, J23, MAPF = _large_inputs(c)
    if metrics is not None:
        GS, J13, J23, MAPF = metrics
    aq = mkinit.aq_props(c.QA) if c.QA else None
    cor = np.zeros((g.IA, g.JA), order="F")
    wd = np.zeros(g.KA)
    st_ref = {n: v.copy(order="F") for n, v in c.state.items()}
    st_gpu = {n: v.copy(order="F") for n, v in c.state.items()}
    out_ref = dict(mflx_hi=g.zeros(3), tflx_hi=g.zeros(3), num_diff=g.zeros(5, 3))
    out_gpu = dict(mflx_hi=g.zeros(3), tflx_hi=g.zeros(3), num_diff=g.zeros(5, 3))
    for _ in range(nlarge):
        oracle.tstep_large(g, c.scheme, c.scheme_tracer, st_ref, out_ref, tp, c.ref, aq, GS, J13, J23, MAPF, cor, wd,
                           c.dtl, c.dt, ND_COEF=c.nd_coef, divdmp=divdmp, fct=c.fct, QA=c.QA, ND_ORDER=nd_order,
                           short=short, tinteg=tinteg)
    lib.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    lib.short_type(short)
    lib.tinteg_short_type(tinteg)
    R, CV, CP, M = aq if aq else (None, None, None, None)
    for _ in range(nlarge):
        lib.ATMOS_DYN_Tstep_large_fvm_heve(
            DENS=st_gpu["DENS"], MOMZ=st_gpu["MOMZ"], MOMX=st_gpu["MOMX"], MOMY=st_gpu["MOMY"], RHOT=st_gpu["RHOT"],
            QTRC=st_gpu.get("QTRC"), QA=c.QA, mflx_hi=out_gpu["mflx_hi"], tflx_hi=out_gpu["tflx_hi"],
            num_diff=out_gpu["num_diff"], RHOQ_tp=tp.get("RHOQ_tp"), CORIOLI=cor, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY,
            FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX,
            RFDY=g.RFDY, PHI=c.ref["PHI"], GSQRT=GS, J13G=J13, J23G=J23, J33G=1.0, MAPF=MAPF, AQ_R=R, AQ_CV=CV,
            AQ_CP=CP, AQ_MASS=M, REF_dens=c.ref["REF_dens"], REF_pott=c.ref["REF_pott"], REF_pres=c.ref["REF_pres"],
            ND_COEF=c.nd_coef, ND_ORDER=nd_order, ND_SFC_FACT=1.0, ND_USE_RS=True, wdamp_coef=wd, divdmp_coef=divdmp,
            FLAG_FCT_TRACER=c.fct, FLAG_FCT_ALONG_STREAM=True, DTLS=c.dtl, DTSS=c.dt,
            **{k: v for k, v in tp.items() if k != "RHOQ_tp"})
    return st_ref, st_gpu


def _field_err(a, b, g):
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    x, y = a[sl], b[sl]
    scale = np.max(np.abs(y))
    return float(np.max(np.abs(x - y)) / scale) if scale > 0 else float(np.max(np.abs(x - y)))


def test_large_step_dry_parity(lib):
    c = mkinit.config(1, scale=0.3)
    st_ref, st_gpu = _run_large_both(c, 4, lib)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"


def test_large_step_higher_order_filter_parity(lib):
    # the numerical filter at ND_ORDER = 2 inside the device large step
    c = mkinit.config(1, scale=0.3)
    st_ref, st_gpu = _run_large_both(c, 2, lib, nd_order=2)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"


def test_large_step_moist_fct_parity(lib):
    c = mkinit.config(2, scale=0.04)
    st_ref, st_gpu = _run_large_both(c, 2, lib)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for iq in range(c.QA):
        err = _field_err(st_gpu["QTRC"][..., iq], st_ref["QTRC"][..., iq], c.g)
        assert err <= 1e-10, f"QTRC[{iq}]: {err:.3e}"


@pytest.mark.parametrize("scheme", ["UD5", "CD6"])
def test_large_step_six_point_schemes_parity(lib, scheme):
    # dynamics and tracers (FCT) with a 6-point scheme, on a lateral halo of 3,
    # through the host-array large step
    g = helpers.small_grid(IMAX=14, JMAX=12, KMAX=20, stretched=True, halo=3)
    c = mkinit.make_case("wide", g, scheme, scheme, dt=1.0, dtl=5.0,
                         bubbles=[(3000.0, 2500.0, 1500.0, 2000.0, 2000.0, 1500.0, 3.0)], theta_noise=0.05,
                         noise_kind="normal", wind_noise=2.0, tracers=2, fct=True, seed=4, u0=3.0, v0=-2.0)
    st_ref, st_gpu = _run_large_both(c, 2, lib, divdmp=0.05)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for iq in range(c.QA):
        err = _field_err(st_gpu["QTRC"][..., iq], st_ref["QTRC"][..., iq], c.g)
        assert err <= 1e-10, f"QTRC[{iq}]: {err:.3e}"


@pytest.mark.parametrize("case", ["dry", "moist_fct"])
def test_large_step_heve_parity(lib, case):
    # the large step with HEVE registered as the short step; being explicit in
    # the vertical, HEVE needs short steps below the vertical acoustic limit
    # dz / c_s (250 m and 50 m lowest layers here)
    c = mkinit.config(1, scale=0.3) if case == "dry" else mkinit.config(2, scale=0.04)
    c.dt, c.dtl = (0.1, 0.5) if case == "dry" else (0.04, 0.2)
    st_ref, st_gpu = _run_large_both(c, 2, lib, short="HEVE")
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for iq in range(c.QA):
        err = _field_err(st_gpu["QTRC"][..., iq], st_ref["QTRC"][..., iq], c.g)
        assert err <= 1e-10, f"QTRC[{iq}]: {err:.3e}"


def test_mass_conserved_on_device(lib):
    import torch

    c = mkinit.config(1, scale=0.4)
    g = c.g
    tp, GS, J13, J23, MAPF = _large_inputs(c)
    lib.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    d = {n: torch.from_numpy(np.ravel(v, order="K").copy()).cuda() for n, v in c.state.items()}
    tpd = {n: torch.from_numpy(np.ravel(v, order="K").copy()).cuda() for n, v in tp.items()}
    refd = {n: torch.from_numpy(np.ravel(v, order="K").copy()).cuda() for n, v in c.ref.items()}
    N3 = int(np.prod(g.shape))
    out = {n: torch.zeros(k * N3, dtype=torch.float64, device="cuda") for n, k in (("mflx_hi", 3), ("tflx_hi", 3), ("num_diff", 15))}
    m0 = lib.domain_sum_dev(d["DENS"], g.CDZ, g.CDX, g.CDY)
    cor = torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda")
    GSd, J13d, J23d, MAPFd = (torch.from_numpy(np.ravel(x, order="K").copy()).cuda() for x in (GS, J13, J23, MAPF))
    for _ in range(10):
        lib.ATMOS_DYN_Tstep_large_fvm_heve_dev(
            DENS=d["DENS"], MOMZ=d["MOMZ"], MOMX=d["MOMX"], MOMY=d["MOMY"], RHOT=d["RHOT"], QTRC=None, QA=0,
            CORIOLI=cor, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX,
            RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY, PHI=refd["PHI"], GSQRT=GSd, J13G=J13d, J23G=J23d,
            J33G=1.0, MAPF=MAPFd, AQ_R=None, AQ_CV=None, AQ_CP=None, AQ_MASS=None, REF_dens=refd["REF_dens"],
            REF_pott=refd["REF_pott"], REF_pres=refd["REF_pres"], ND_COEF=c.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0,
            ND_USE_RS=True, wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0, FLAG_FCT_TRACER=False,
            FLAG_FCT_ALONG_STREAM=True, DTLS=c.dtl, DTSS=c.dt, RHOQ_tp=None, **out, **tpd)
    lib.check()
    m1 = lib.domain_sum_dev(d["DENS"], g.CDZ, g.CDX, g.CDY)
    assert abs(m1 - m0) / m0 < 1e-13, (m0, m1)


def test_single_terrain_point_takes_the_metric_stage(lib):
    # one GSQRT value off 1 is terrain: the HEVI stage runs the general-metric
    # kernels, bit-exact with the oracle
    g = helpers.small_grid()
    c = helpers.small_case(g)
    a = helpers.short_inputs(c, full=False)
    a["GSQRT"] = a["GSQRT"].copy(order="F")
    a["GSQRT"][3, 4, 5, 0] = 1.01
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short(g, "UD3", o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_call_args(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), n


def test_nonperiodic_boundary_is_rejected(lib):
    g = helpers.small_grid()
    c = helpers.small_case(g)
    a = helpers.short_inputs(c, full=False)
    kw = _stage_call_args(a, helpers.stage_outputs(g))
    kw["BND_W"] = True
    lib.setup(g.index_dict(), "UD3", "UD3")
    with pytest.raises(hevi.HeviError) as e:
        lib.ATMOS_DYN_Tstep_short_fvm_hevi(**kw)
    assert e.value.code == 5


def test_nonfinite_input_raises(lib):
    g = helpers.small_grid()
    c = helpers.small_case(g)
    a = helpers.short_inputs(c, full=False)
    a["RHOT"] = a["RHOT"].copy(order="F")
    a["RHOT"][6, 5, 5] = np.nan
    lib.setup(g.index_dict(), "UD3", "UD3")
    with pytest.raises(hevi.HeviError) as e:
        lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_call_args(a, helpers.stage_outputs(g, 0.0)))
    assert e.value.code == 4


def test_warm_bubble_600_short_steps(lib):
    """The 40x40x80 UD3 warm bubble (dx = dy = 500 m, dz = 250 m, dt = 1 s) over
    600 short steps (120 large steps of 5): every prognostic field within 1e-10
    of the oracle, relative to the field's largest magnitude, and the domain
    mass conserved to round-off on both sides (the oracle itself drifts by
    about 2e-13 over the run: flux-form updates, 128 000 cells, 600 steps)."""
    c = mkinit.config(1)
    g = c.g
    m0 = oracle.domain_sum(g, c.state["DENS"])
    st_ref, st_gpu = _run_large_both(c, 120, lib)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for st in (st_ref, st_gpu):
        m1 = oracle.domain_sum(g, st["DENS"])
        assert abs(m1 - m0) / m0 < 1e-12


@pytest.mark.parametrize("stretched", [False, True])
def test_divergence_bit_exact(lib, stretched):
    g = helpers.small_grid(IMAX=13, JMAX=11, KMAX=17, stretched=stretched)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    ref = np.full(g.shape, np.nan, order="F")
    oracle.divergence(g, ref, c.state, GS, J13, J23, 1.0, MAPF)
    got = np.full(g.shape, np.nan, order="F")
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_divergence(DDIV=got, MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"], MOMY=c.state["MOMY"], GSQRT=GS,
                             J13G=J13, J23G=J23, J33G=1.0, MAPF=MAPF, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY,
                             RFDZ=g.RFDZ, FDZ=g.FDZ)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


def test_large_step_with_divergence_damping(lib):
    c = mkinit.config(1, scale=0.3)
    st_ref, st_gpu = _run_large_both(c, 3, lib, divdmp=0.1)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
