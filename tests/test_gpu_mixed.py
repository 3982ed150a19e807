"""The mixed-precision short step (FP32 flux arithmetic, FP64 state and
vertical solve) against the plain FP64 path on the same inputs: the error of
every prognostic field after many short steps stays within the bound the
mixed path is specified to (1e-5 of the field's largest magnitude), and the
FP64 path itself is untouched by the templating (checked bit for bit against
the oracle in test_gpu_parity)."""
import numpy as np
import pytest

from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


def run_short_steps(c, nsteps, mixed, hook=False):
    """nsteps short steps (numfilter + RK4 + boundary values and halo) on the
    device, FP64 or mixed; returns the final state on the host. hook: the
    halo fills go through a 1x1 decomposition's exchange (scale_b200.decomp)."""
    import torch

    g = c.g
    N3 = int(np.prod(g.shape))
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    dev = lambda x: torch.from_numpy(np.ravel(x, order="K").copy()).cuda()  # noqa: E731
    X = {n: dev(c.state[n]) for n in STATE}
    ft = torch.float32 if mixed else torch.float64
    z = lambda k=1: torch.zeros(k * N3, dtype=ft, device="cuda")  # noqa: E731
    mflx, tflx, nd = z(3), z(3), z(15)
    tend = {n: z() for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")}
    ref = {n: dev(v) for n, v in c.ref.items()}
    dp0, rt2p, refr = dev(DPRES0), dev(RT2P), dev(REF_rhot)
    GS = torch.ones(7 * N3, dtype=torch.float64, device="cuda")
    J0 = torch.zeros(7 * N3, dtype=torch.float64, device="cuda")
    MAPF = torch.ones(g.IA * g.JA * 8, dtype=torch.float64, device="cuda")
    cor = torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda")
    grid = dict(CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ,
                RFDX=g.RFDX, RFDY=g.RFDY)
    nf = hevi.ATMOS_DYN_numfilter_coef_mixed_dev if mixed else hevi.ATMOS_DYN_numfilter_coef_dev
    rk = hevi.ATMOS_DYN_Tinteg_short_rk4_mixed_dev if mixed else hevi.ATMOS_DYN_Tinteg_short_rk4_dev
    hevi.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    if hook:
        from scale_b200 import decomp

        decomp.attach(hevi, decomp.Decomposition(g.IMAX, g.JMAX, 1, 1, 0, g.halo), g.KA)
    try:
        for _ in range(nsteps):
            nf(num_diff=nd, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=c.dt,
               REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"], ND_COEF=c.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0,
               ND_USE_RS=True, **X)
            rk(PROG=None, mflx_hi=mflx, tflx_hi=tflx, DPRES0=dp0, RT2P=rt2p, CORIOLI=cor, num_diff=nd,
               wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0, DDIV=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
               FLAG_FCT_ALONG_STREAM=True, PHI=ref["PHI"], GSQRT=GS, J13G=J0, J23G=J0, J33G=1.0, MAPF=MAPF,
               REF_dens=ref["REF_dens"], REF_rhot=refr, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=c.dt,
               **X, **tend, **grid)
            hevi.boundary_dev(**X)
        hevi.check()
        return {n: X[n].cpu().numpy().reshape(g.shape, order="F") for n in STATE}
    finally:
        hevi.finalize()


def field_errors(a, b, g):
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    x, y = a[sl], b[sl]
    scale = np.max(np.abs(y))
    d = np.abs(x - y)
    return float(d.max() / scale), float(np.sqrt(np.mean(d * d)) / scale)


def test_mixed_precision_error_after_600_short_steps():
    # the 1024x1024x96 multi-bubble configuration on a 64x64 horizontal patch
    c = mkinit.config(4, scale=1 / 16)
    st64 = run_short_steps(c, 600, mixed=False)
    st32 = run_short_steps(c, 600, mixed=True)
    for n in STATE:
        emax, erms = field_errors(st32[n], st64[n], c.g)
        assert emax <= 1e-5, f"{n}: max {emax:.3e} rms {erms:.3e}"
        assert np.isfinite(st32[n]).all()


def test_mixed_precision_conserves_mass():
    c = mkinit.config(4, scale=1 / 16)
    import oracle

    m0 = oracle.domain_sum(c.g, c.state["DENS"])
    st32 = run_short_steps(c, 50, mixed=True)
    m1 = oracle.domain_sum(c.g, st32["DENS"])
    # the flux-form update telescopes, but the FP32 flux differences round
    # (about 1e-10 of the density per cell and step, random in sign)
    drift = abs(m1 - m0) / m0
    print(f"mixed-precision mass drift after 50 short steps: {drift:.3e}")
    assert drift < 1e-8


@pytest.mark.parametrize("scheme", ["UD5", "CD6"])
def test_mixed_precision_six_point_schemes(scheme):
    # a warm bubble on a lateral halo of 3, 100 short steps, FP32 fluxes against FP64
    g = mkinit.uniform_grid(32, 32, 32, 200.0, 200.0, 200.0, halo=3)
    c = mkinit.make_case("mixed six-point", g, scheme, scheme, dt=0.4, dtl=2.0,
                         bubbles=[(3200.0, 3200.0, 2000.0, 1500.0, 1500.0, 1000.0, 2.0)], theta_noise=0.01, seed=7)
    st64 = run_short_steps(c, 100, mixed=False)
    st32 = run_short_steps(c, 100, mixed=True)
    for n in STATE:
        emax, erms = field_errors(st32[n], st64[n], c.g)
        assert emax <= 1e-5, f"{n}: max {emax:.3e} rms {erms:.3e}"


@pytest.mark.parametrize("fct,along", [(False, True), (True, True), (True, False)])
def test_mixed_tracer_rk3_matches_fp64(fct, along):
    """The tracer RK3 with FP32 flux and limiter arithmetic against the FP64
    entry on the same inputs (the FP32 mass fluxes, num_diff and tendency are
    the FP64 ones rounded): the tracer agrees to 1e-5 of its largest value and
    the limiter keeps it as bounded as the FP64 limiter does."""
    import torch

    import helpers
    from test_gpu_parity import _tracer_inputs

    g = helpers.small_grid(IMAX=20, JMAX=16, KMAX=24, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, _, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ndq = np.asfortranarray(1e-6 * np.random.default_rng(9).normal(size=g.shape + (3,)))
    dev = lambda x, t=torch.float64: torch.from_numpy(np.ravel(x, order="K").copy()).to("cuda", t)  # noqa: E731
    out = {}
    hevi.setup(g.index_dict(), "UD3", "UD3")

    def run(mixed):
        ft = torch.float32 if mixed else torch.float64
        q = dev(q0)
        kw = dict(QTRC=q, QTRC0=q, RHOQ_t=dev(rhoq, ft), DENS0=dev(d0), DENS=dev(d), mflx_hi=dev(mflx, ft),
                  num_diff=dev(ndq, ft), GSQRT=dev(GS), MAPF=dev(MAPF), CDZ=g.CDZ, RCDZ=g.RCDZ, RCDX=g.RCDX,
                  RCDY=g.RCDY, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dtl=5.0,
                  FLAG_FCT_TRACER=fct, FLAG_FCT_ALONG_STREAM=along)
        for _ in range(3):
            (hevi.ATMOS_DYN_Tinteg_tracer_rk3_mixed_dev if mixed else hevi.ATMOS_DYN_Tinteg_tracer_rk3_dev)(**kw)
            hevi.COMM_vars8_dev(q, 1)
        hevi.check()
        return q.cpu().numpy().reshape(g.shape, order="F")

    try:
        for mixed in (False, True):
            out[mixed] = run(mixed)
        # the three-kernel limiter in FP32 (FMA contractions may differ from the fused form's)
        hevi.tracer_fct_form(False)
        out["three_kernel"] = run(True)
    finally:
        hevi.finalize()
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    a64, a32 = out[False][sl], out[True][sl]
    assert np.isfinite(a32).all()
    err = np.max(np.abs(a32 - a64)) / np.max(np.abs(a64))
    assert err <= 1e-5, f"max relative error {err:.3e}"
    err3 = np.max(np.abs(out["three_kernel"][sl] - a32)) / np.max(np.abs(a64))
    assert err3 <= 1e-6, f"fused against three-kernel FP32 limiter: {err3:.3e}"
    if fct:
        # no new minimum beyond FP32 rounding of the FP64 run's own
        assert a32.min() >= a64.min() - 1e-6 * np.max(np.abs(a64))


def test_mixed_numfilter_tiled_form_matches_column_form():
    """The FP32 filter from staged tiles against the FP32 column kernel on the
    same inputs (two FP32 builds: FMA contraction may differ, so to 1e-6 of
    each component's largest value)."""
    import torch

    import helpers

    g = helpers.small_grid(IMAX=13, JMAX=10, KMAX=36, stretched=True)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    dev = lambda x: torch.from_numpy(np.ravel(x, order="K").copy()).cuda()  # noqa: E731
    out = []
    for tiled in (True, False):
        hevi.setup(g.index_dict(), "UD3", "UD3")
        try:
            hevi.numfilter_form(tiled)
            nd = torch.zeros(15 * int(np.prod(g.shape)), dtype=torch.float32, device="cuda")
            hevi.ATMOS_DYN_numfilter_coef_mixed_dev(
                num_diff=nd, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5,
                REF_dens=dev(c.ref["REF_dens"]), REF_pott=dev(c.ref["REF_pott"]), ND_COEF=1e-3, ND_ORDER=1,
                ND_SFC_FACT=0.7, ND_USE_RS=True, **{n: dev(c.state[n]) for n in STATE})
            hevi.check()
            out.append(nd.cpu().numpy().reshape(g.shape + (15,), order="F"))
        finally:
            hevi.finalize()
    for q in range(15):
        scale = np.max(np.abs(out[1][..., q]))
        assert np.max(np.abs(out[0][..., q] - out[1][..., q])) <= 1e-6 * max(scale, 1e-30), q
