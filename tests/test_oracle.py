"""The oracle pinned by the reference's own tests of this path.

The reference ships no golden vectors for the HEVI short step. Its tests are
property tests (scalelib/test/unit/test_atmos_dyn.f90:307-763), the halo test
(scalelib/test/unit/test_comm.f90:150-250) and the DEBUG self-check of the
implicit solve (scale_atmos_dyn_tstep_short_fvm_hevi.F90:1131-1271). They are
re-run here on the oracle with the HEVI scheme.
"""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import mkinit

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


def _large(c, nlarge=1, fct=None, qa=None):
    g = c.g
    QA = c.QA if qa is None else qa
    tp = {n: g.zeros() for n in ("DENS_tp", "MOMZ_tp", "MOMX_tp", "MOMY_tp", "RHOT_tp")}
    if QA:
        tp["RHOQ_tp"] = g.zeros(QA)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    out = dict(mflx_hi=g.zeros(3), tflx_hi=g.zeros(3), num_diff=g.zeros(5, 3))
    aq = mkinit.aq_props(QA) if QA else None
    for _ in range(nlarge):
        oracle.tstep_large(g, c.scheme, c.scheme_tracer, c.state, out, tp, c.ref, aq, GS, J13, J23, MAPF,
                           np.zeros((g.IA, g.JA), order="F"), np.zeros(g.KA), c.dtl, c.dt, ND_COEF=c.nd_coef,
                           fct=c.fct if fct is None else fct, QA=QA)
    return out


def _interior(a, g):
    return a[g.KS - 1 : g.KE, g.IS - 1 : g.IE, g.JS - 1 : g.JE]


SCHEMES = ["UD3", "CD4", "UD3KOREN1993", "CD2", "UD5", "CD6"]


@pytest.mark.parametrize("scheme", SCHEMES)
def test_const(scheme):
    """test_const (test_atmos_dyn.f90:382-454): a horizontally uniform state stays uniform."""
    g = helpers.small_grid(8, 6, 12, halo=helpers.halo_of(scheme))
    c = mkinit.make_case("const", g, scheme, scheme, tracers=1, fct=True)
    st = c.state
    st["DENS"][...] = 1.0
    st["MOMZ"][...] = 2.0
    st["MOMX"][...] = 3.0
    st["MOMY"][...] = 4.0
    st["RHOT"][...] = 300.0
    st["QTRC"][...] = 0.1
    mkinit.vertical_fill(st, g)
    c.ref["REF_dens"][...] = 1.0
    c.ref["REF_pott"][...] = 300.0
    c.ref["REF_pres"][...] = 1000.0
    c.dtl, c.dt = 1.0, 1.0
    _large(c)
    for n in STATE:
        x = _interior(st[n], g)
        assert np.array_equal(x, np.broadcast_to(x[:, :1, :1], x.shape)), n
    q = _interior(st["QTRC"][..., 0], g)
    assert np.array_equal(q, np.broadcast_to(q[:, :1, :1], q.shape))


@pytest.mark.parametrize("scheme", SCHEMES)
def test_conserve(scheme):
    """test_conserve (test_atmos_dyn.f90:456-592): domain totals of DENS and RHOT
    (weighted by the cell volume) are conserved to round-off."""
    g = helpers.small_grid(10, 8, 14, stretched=True, halo=helpers.halo_of(scheme))
    c = mkinit.make_case("conserve", g, scheme, scheme)
    k, i, j = np.meshgrid(np.arange(1, g.KA + 1), np.arange(1, g.IA + 1), np.arange(1, g.JA + 1), indexing="ij")
    st = c.state
    st["MOMZ"][...] = (k + i + j) * 0.1
    st["MOMX"][...] = (k * 2 + i + j) * 0.1
    st["MOMY"][...] = (k + i * 2 + j) * 0.1
    st["DENS"][...] = c.ref["REF_dens"] + (k * 2 + i * 2 + j) * 1e-3
    st["RHOT"][...] = st["DENS"] * (300.0 + (k + i + j * 2) * 0.01)
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    m0 = oracle.domain_sum(g, st["DENS"])
    t0 = oracle.domain_sum(g, st["RHOT"])
    _large(c, 2)
    assert abs(oracle.domain_sum(g, st["DENS"]) - m0) / m0 < 1e-13
    assert abs(oracle.domain_sum(g, st["RHOT"]) - t0) / t0 < 1e-13


@pytest.mark.parametrize("scheme", ["UD3", "UD5", "CD6"])
def test_cwc(scheme):
    """test_cwc (test_atmos_dyn.f90:594-670): uniform theta and tracer stay uniform
    under random momenta (consistency with the continuity equation)."""
    g = helpers.small_grid(10, 10, 14, halo=helpers.halo_of(scheme))
    c = mkinit.make_case("cwc", g, scheme, scheme, tracers=1, fct=True)
    rng = np.random.Generator(np.random.PCG64(3))
    st = c.state
    st["DENS"][...] = c.ref["REF_dens"] * (1.0 + 1e-3 * rng.uniform(-1, 1, size=g.shape))
    st["MOMZ"][...] = rng.uniform(-1, 1, size=g.shape)
    st["MOMX"][...] = rng.uniform(-3, 3, size=g.shape)
    st["MOMY"][...] = rng.uniform(-3, 3, size=g.shape)
    st["RHOT"][...] = st["DENS"] * 300.0
    st["QTRC"][...] = 0.01
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    c.ref["REF_pott"][...] = 300.0
    _large(c)
    pott = _interior(st["RHOT"] / st["DENS"], g)
    assert np.max(np.abs(pott - 300.0)) / 300.0 < 1e-12
    q = _interior(st["QTRC"][..., 0], g)
    assert np.max(np.abs(q - 0.01)) / 0.01 < 1e-12


@pytest.mark.parametrize("along", [True, False])
def test_fct_minmax(along):
    """test_fctminmax (test_atmos_dyn.f90:672-763): with FCT the tracer stays
    inside its initial range."""
    g = helpers.small_grid(12, 12, 16)
    c = helpers.small_case(g, "UD3", tracers=1, wind=5.0)
    c.fct = True
    rng = np.random.Generator(np.random.PCG64(9))
    q = c.state["QTRC"]
    q[..., 0] = np.where(rng.uniform(size=g.shape) > 0.5, 1.0e-3, 0.0)
    mkinit.periodic_fill(q[..., 0], g)
    qmin, qmax = 0.0, 1.0e-3
    GS, _, _, MAPF = oracle.flat_metrics(g)
    tp = {n: g.zeros() for n in ("DENS_tp", "MOMZ_tp", "MOMX_tp", "MOMY_tp", "RHOT_tp")}
    tp["RHOQ_tp"] = g.zeros(1)
    out = dict(mflx_hi=g.zeros(3), tflx_hi=g.zeros(3), num_diff=g.zeros(5, 3))
    for _ in range(2):
        oracle.tstep_large(g, "UD3", "UD3", c.state, out, tp, c.ref, mkinit.aq_props(1), GS, *oracle.flat_metrics(g)[1:3],
                           MAPF, np.zeros((g.IA, g.JA), order="F"), np.zeros(g.KA), 5.0, 1.0, fct=True, along=along, QA=1)
    x = _interior(q[..., 0], g)
    eps = 1e-10
    assert x.min() >= qmin - eps and x.max() <= qmax * (1.0 + eps)


def test_no_undefined_values_leak():
    """test_undef (test_atmos_dyn.f90:307-380): NaN in the vertical halo of the
    state never reaches the interior (the short step reads only defined cells)."""
    g = helpers.small_grid(10, 8, 14)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    for n in STATE:
        c.state[n][: g.KS - 1] = np.nan
        c.state[n][g.KE :] = np.nan
    _large(c, 1)
    for n in STATE:
        assert np.all(np.isfinite(_interior(c.state[n], g))), n


def test_solver_residual_check():
    """check_equation (tstep_short_fvm_hevi.F90:1131-1271) aborts above 1e-6; it
    was written for CD4 face values and uniform dz."""
    g = helpers.small_grid(10, 10, 20)
    c = helpers.small_case(g, "CD4")
    helpers.perturb_state(c)
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    nd = g.zeros(5, 3)
    oracle.numfilter(g, nd, c.state, c.ref, DT=1.0)
    r = oracle.max_residual(g, "CD4", c.state, DPRES0, RT2P, nd, c.ref, REF_rhot, 0.5)
    assert r < 1e-6


def test_halo_fill_neighbours():
    """test_comm.f90:150-250: the N/S/E/W and corner halos hold the periodic neighbours."""
    g = helpers.small_grid(7, 5, 6)
    k, i, j = np.meshgrid(np.arange(1, g.KA + 1), np.arange(1, g.IA + 1), np.arange(1, g.JA + 1), indexing="ij")
    a = np.asfortranarray((k * 10000 + i * 100 + j).astype(np.float64))
    oracle.halo(g, a)
    wi = lambda ii: ii + g.IMAX if ii < g.IS else (ii - g.IMAX if ii > g.IE else ii)  # noqa: E731
    wj = lambda jj: jj + g.JMAX if jj < g.JS else (jj - g.JMAX if jj > g.JE else jj)  # noqa: E731
    for ii in range(1, g.IA + 1):
        for jj in range(1, g.JA + 1):
            exp = np.arange(1, g.KA + 1) * 10000 + wi(ii) * 100 + wj(jj)
            assert np.array_equal(a[:, ii - 1, jj - 1], exp), (ii, jj)
    b = a.copy(order="F")
    mkinit.periodic_fill(b, g)
    assert np.array_equal(a, b)


def test_rk4_equals_four_stages():
    """ATMOS_DYN_tinteg_short_rk4 restated twice: the oracle's integrator against
    an explicit sequence of four oracle stages plus the combine (rk4.F90:376-650)."""
    g = helpers.small_grid(9, 8, 12)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for kk in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(kk)
    x = {n: c.state[n].copy(order="F") for n in STATE}
    x["mflx_hi"] = g.zeros(3)
    x["tflx_hi"] = g.zeros(3)
    x0 = {n: v.copy(order="F") for n, v in x.items()}
    oracle.tinteg_short_rk4(g, "UD3", x, dict(a, dt=1.0))
    rk, fl = [], []
    cur = {n: x0[n] for n in STATE}
    for s, dtrk in enumerate((0.5, 0.5, 1.0, 1.0)):
        o = helpers.stage_outputs(g, 0.0)
        args = dict(a, dtrk=dtrk)
        args.update({n + "0": x0[n] for n in STATE})
        args.update(cur)
        if s == 3:
            o["mflx_hi"] = x0["mflx_hi"].copy(order="F")
            o["tflx_hi"] = x0["tflx_hi"].copy(order="F")
        oracle.tstep_short(g, "UD3", o, args)
        st = {n: o[n + "_RK"] for n in STATE}
        if s < 3:
            for n in STATE:
                oracle.halo(g, st[n])
        rk.append(st)
        fl.append((o["mflx_hi"], o["tflx_hi"]))
        cur = st
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    for n in STATE:
        exp = (rk[0][n] * 2.0 + rk[1][n] * 4.0 + rk[2][n] * 2.0 + rk[3][n] - x0[n] * 3.0) / 6.0
        ks = slice(g.KS - 1, g.KE - 1) if n == "MOMZ" else sl[0]
        assert np.array_equal(x[n][ks, sl[1], sl[2]], exp[ks, sl[1], sl[2]]), n
    for f in range(2):
        exp = (fl[0][f] + fl[1][f] * 2.0 + fl[2][f] * 2.0 + fl[3][f]) / 6.0
        got = x["mflx_hi" if f == 0 else "tflx_hi"]
        assert np.array_equal(got[sl], exp[sl])


@pytest.mark.parametrize("ws2002", [True, False])
def test_rk3_equals_three_stages(ws2002):
    """ATMOS_DYN_tinteg_short_rk3 restated twice: the oracle's integrator against
    an explicit sequence of three oracle stages, with Heun's combine for RK3
    (scale_atmos_dyn_tinteg_short_rk3.F90:188-576)."""
    g = helpers.small_grid(9, 8, 12)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for kk in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(kk)
    x = {n: c.state[n].copy(order="F") for n in STATE}
    x["mflx_hi"] = g.zeros(3) + 7.0
    x["tflx_hi"] = g.zeros(3) + 7.0
    x0 = {n: v.copy(order="F") for n, v in x.items()}
    dt = 1.5
    oracle.tinteg_short_rk3(g, "CD4", x, dict(a, dt=dt), ws2002=ws2002)
    rk, fl = [], []
    cur = {n: x0[n] for n in STATE}
    for s, dtrk in enumerate((dt * (1.0 / 3.0), dt * (1.0 / 2.0 if ws2002 else 2.0 / 3.0), dt)):
        o = helpers.stage_outputs(g, 0.0)
        args = dict(a, dtrk=dtrk)
        args.update({n + "0": x0[n] for n in STATE})
        args.update(cur)
        if s == 2:
            o["mflx_hi"] = x0["mflx_hi"].copy(order="F")
            o["tflx_hi"] = x0["tflx_hi"].copy(order="F")
        oracle.tstep_short(g, "CD4", o, args)
        st = {n: o[n + "_RK"] for n in STATE}
        if s < 2:
            for n in STATE:
                oracle.halo(g, st[n])
        rk.append(st)
        fl.append((o["mflx_hi"], o["tflx_hi"]))
        cur = st
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    for n in STATE:
        exp = rk[2][n] if ws2002 else (rk[0][n] * 3.0 + rk[2][n] * 3.0 - x0[n] * 2.0) / 4.0
        ks = slice(g.KS - 1, g.KE - 1) if n == "MOMZ" else sl[0]
        assert np.array_equal(x[n][ks, sl[1], sl[2]], exp[ks, sl[1], sl[2]]), n
    for f in range(2):
        got = x["mflx_hi" if f == 0 else "tflx_hi"]
        exp = fl[2][f] if ws2002 else (fl[0][f] + fl[2][f] * 3.0) / 4.0
        assert np.array_equal(got[sl], exp[sl])


@pytest.mark.parametrize("tinteg", ["RK3", "RK3WS2002"])
def test_rk3_conserve(tinteg):
    """test_conserve (test_atmos_dyn.f90:456-592) with the RK3 short integrators:
    the volume-weighted totals of DENS and RHOT are conserved to round-off."""
    g = helpers.small_grid(10, 8, 14, stretched=True)
    c = mkinit.make_case("conserve rk3", g, "CD4", "CD4", dt=0.5)
    k, i, j = np.meshgrid(np.arange(1, g.KA + 1), np.arange(1, g.IA + 1), np.arange(1, g.JA + 1), indexing="ij")
    st = c.state
    st["MOMZ"][...] = (k + i + j) * 0.01
    st["MOMX"][...] = (k * 2 + i + j) * 0.01
    st["MOMY"][...] = (k + i * 2 + j) * 0.01
    st["DENS"][...] = c.ref["REF_dens"] + (k * 2 + i * 2 + j) * 1e-4
    st["RHOT"][...] = st["DENS"] * (300.0 + (k + i + j * 2) * 0.01)
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    m0 = oracle.domain_sum(g, st["DENS"])
    t0 = oracle.domain_sum(g, st["RHOT"])
    a = helpers.short_inputs(c, full=False)
    for kk in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(kk)
    x = {n: st[n] for n in STATE}
    x["mflx_hi"], x["tflx_hi"] = g.zeros(3), g.zeros(3)
    for _ in range(3):
        oracle.tinteg_short_rk3(g, c.scheme, x, dict(a, dt=c.dt), ws2002=(tinteg == "RK3WS2002"))
        for n in STATE:
            mkinit.periodic_fill(st[n], g)
        mkinit.vertical_fill(st, g)
    assert abs(oracle.domain_sum(g, st["DENS"]) - m0) / m0 < 1e-13
    assert abs(oracle.domain_sum(g, st["RHOT"]) - t0) / t0 < 1e-13


def _periodic_metrics(g, seed, amp=0.05):
    """Seeded terrain-following metrics, periodic across the lateral halo."""
    rng = np.random.Generator(np.random.PCG64(seed))
    GS = np.asfortranarray(1.0 + amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    J13 = np.asfortranarray(amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    J23 = np.asfortranarray(amp * rng.uniform(-1, 1, size=g.shape + (7,)))
    for arr in (GS, J13, J23):
        for q in range(7):
            mkinit.periodic_fill(arr[..., q], g)
    MAPF = np.asfortranarray(1.0 + amp * rng.uniform(-1, 1, size=(g.IA, g.JA, 2, 4)))
    for a in range(2):
        for b in range(4):
            mkinit.periodic_fill(MAPF[None, :, :, a, b], g)
    return GS, J13, J23, MAPF


@pytest.mark.parametrize("short", ["HEVI", "HEVE"])
def test_terrain_conserve(short):
    """test_conserve (test_atmos_dyn.f90:456-592) with terrain-following
    metrics: the total mass sum(DENS * GSQRT / (MAPF_1 * MAPF_2) * volume),
    the quantity the flux form of Sr (tstep_short_fvm_hevi.F90:443-479)
    telescopes, is conserved to round-off by the oracle's short steps."""
    g = helpers.small_grid(10, 8, 14, stretched=True)
    c = mkinit.make_case("conserve terrain", g, "CD4", "CD4", dt=0.2 if short == "HEVI" else 0.05)
    k, i, j = np.meshgrid(np.arange(1, g.KA + 1), np.arange(1, g.IA + 1), np.arange(1, g.JA + 1), indexing="ij")
    st = c.state
    st["MOMZ"][...] = (k + i + j) * 0.01
    st["MOMX"][...] = (k * 2 + i + j) * 0.01
    st["MOMY"][...] = (k + i * 2 + j) * 0.01
    st["DENS"][...] = c.ref["REF_dens"] + (k * 2 + i * 2 + j) * 1e-4
    st["RHOT"][...] = st["DENS"] * (300.0 + (k + i + j * 2) * 0.01)
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    GS, J13, J23, MAPF = _periodic_metrics(g, 9)
    w = GS[..., 0] / (MAPF[:, :, 0, 0] * MAPF[:, :, 1, 0])[None, :, :]

    def total(x):
        return oracle.domain_sum(g, np.asfortranarray(x * w))

    m0, t0 = total(st["DENS"]), total(st["RHOT"])
    a = helpers.short_inputs(c, full=False)
    for kk in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(kk)
    a.update(GSQRT=GS, J13G=J13, J23G=J23, MAPF=MAPF)
    x = {n: st[n] for n in STATE}
    x["mflx_hi"], x["tflx_hi"] = g.zeros(3), g.zeros(3)
    for _ in range(3):
        oracle.tinteg_short_rk4(g, c.scheme, x, dict(a, dt=c.dt), short=short)
        for n in STATE:
            mkinit.periodic_fill(st[n], g)
        mkinit.vertical_fill(st, g)
    assert abs(total(st["DENS"]) - m0) / m0 < 1e-13
    assert abs(total(st["RHOT"]) - t0) / t0 < 1e-13


@pytest.mark.parametrize("fct", [False, True])
def test_koren_tracer_keeps_uniform_tracer(fct):
    """test_cwc with the UD3KOREN1993 tracer flux (the reference's default
    tracer scheme): a uniform tracer stays uniform under random momenta."""
    g = helpers.small_grid(10, 10, 14)
    c = mkinit.make_case("cwc koren", g, "UD3", "UD3KOREN1993", tracers=1, fct=fct)
    rng = np.random.Generator(np.random.PCG64(5))
    st = c.state
    st["DENS"][...] = c.ref["REF_dens"] * (1.0 + 1e-3 * rng.uniform(-1, 1, size=g.shape))
    st["MOMZ"][...] = rng.uniform(-1, 1, size=g.shape)
    st["MOMX"][...] = rng.uniform(-3, 3, size=g.shape)
    st["MOMY"][...] = rng.uniform(-3, 3, size=g.shape)
    st["RHOT"][...] = st["DENS"] * 300.0
    st["QTRC"][...] = 0.01
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    c.ref["REF_pott"][...] = 300.0
    _large(c)
    q = _interior(st["QTRC"][..., 0], g)
    assert np.max(np.abs(q - 0.01)) / 0.01 < 1e-12


def _step_advection(scheme, g, cfl=0.2):
    """One tracer stage of a step function in x under a uniform x mass flux."""
    q = g.zeros()
    x = np.arange(g.IA)
    q[:, (x >= g.IS - 1 + g.IMAX // 4) & (x < g.IS - 1 + g.IMAX // 2), :] = 1.0
    mkinit.periodic_fill(q, g)
    d = np.asfortranarray(np.ones(g.shape))
    mflx = g.zeros(3)
    mflx[..., 1] = 1.0
    dtl = cfl * g.DX
    GS, _, _, MAPF = oracle.flat_metrics(g)
    out = np.full(g.shape, np.nan, order="F")
    oracle.tstep_tracer(g, scheme, out, q, q, g.zeros(), d, d, mflx, g.zeros(3), GS, np.asfortranarray(MAPF[..., 0]),
                        dtl, False, True)
    return _interior(out, g)


def test_koren_limiter_keeps_step_bounded():
    """The Koren (1993) limiter is total-variation diminishing: advecting a
    step function with UD3KOREN1993 (no FCT) creates no new extrema, while the
    unlimited UD3 flux over- and undershoots."""
    g = helpers.small_grid(32, 4, 6)
    qk = _step_advection("UD3KOREN1993", g)
    assert qk.min() >= -1e-15 and qk.max() <= 1.0 + 1e-15
    qu = _step_advection("UD3", g)
    assert qu.min() < -1e-3 or qu.max() > 1.0 + 1e-3


def test_numfilter_higher_orders_damp_the_two_grid_wave_alike():
    """The filter coefficient DIFF4 * dx**(4*order) / 2**(4*order) normalises
    every order (calc_numdiff with calc_diff4, scale_atmos_dyn_common.F90:
    444-460, 1518-1918) so that a 2-dx wave is damped the same: for a density
    anomaly alternating along x on a uniform grid, num_diff(DENS, x) agrees
    for ND_ORDER 1, 2 and 3; a uniform state gives zero at every order."""
    g = mkinit.uniform_grid(16, 8, 12, 500.0, 500.0, 250.0)
    c = mkinit.make_case("2dx", g, "UD3", "UD3")
    st = c.state
    i = np.arange(g.IA)
    st["DENS"][...] = c.ref["REF_dens"] + 1e-3 * np.where(i % 2 == 0, 1.0, -1.0)[None, :, None]
    st["RHOT"][...] = st["DENS"] * c.ref["REF_pott"]
    for n in ("MOMZ", "MOMX", "MOMY"):
        st[n][...] = 0.0
    out = {}
    for order in (1, 2, 3):
        nd = g.zeros(5, 3)
        assert oracle.numfilter(g, nd, st, c.ref, DT=1.0, ND_COEF=1e-2, ND_ORDER=order) == 0
        out[order] = _interior(nd[..., 0, 1], g)
    scale = np.max(np.abs(out[1]))
    assert scale > 0.0
    for order in (2, 3):
        assert np.max(np.abs(out[order] - out[1])) <= 1e-12 * scale, order
    # uniform state: no diffusion at any order
    st["DENS"][...] = c.ref["REF_dens"]
    st["RHOT"][...] = st["DENS"] * c.ref["REF_pott"]
    for order in (2, 3):
        nd = g.zeros(5, 3)
        oracle.numfilter(g, nd, st, c.ref, DT=1.0, ND_COEF=1e-2, ND_ORDER=order)
        assert np.max(np.abs(_interior(nd[..., 0, 1], g))) < 1e-14


def _heve_steps(c, nsteps):
    """nsteps RK4 short steps with the HEVE stage; c.state is advanced in place."""
    g = c.g
    a = helpers.short_inputs(c, full=False)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    x = {n: c.state[n] for n in STATE}
    x["mflx_hi"], x["tflx_hi"] = g.zeros(3), g.zeros(3)
    for _ in range(nsteps):
        oracle.tinteg_short_rk4(g, c.scheme, x, dict(a, dt=c.dt), short="HEVE")
        for n in STATE:  # the large step's halo fill after each short step
            mkinit.periodic_fill(c.state[n], g)
        mkinit.vertical_fill(c.state, g)
    return x


@pytest.mark.parametrize("scheme", ["UD3", "CD4", "UD5"])
def test_heve_const(scheme):
    """test_const (test_atmos_dyn.f90:382-454) with the HEVE short step: a
    horizontally uniform state stays uniform."""
    g = helpers.small_grid(8, 6, 12, halo=helpers.halo_of(scheme))
    c = mkinit.make_case("const heve", g, scheme, scheme, dt=0.5)
    st = c.state
    st["DENS"][...] = c.ref["REF_dens"]
    st["MOMX"][...] = 3.0
    st["MOMY"][...] = 4.0
    st["RHOT"][...] = c.ref["REF_dens"] * 300.0
    st["MOMZ"][...] = 0.0
    mkinit.vertical_fill(st, g)
    _heve_steps(c, 3)
    for n in STATE:
        x = _interior(st[n], g)
        assert np.array_equal(x, np.broadcast_to(x[:, :1, :1], x.shape)), n
        assert np.isfinite(x).all(), n


@pytest.mark.parametrize("scheme", ["UD3", "CD4", "UD5"])
def test_heve_conserve(scheme):
    """test_conserve (test_atmos_dyn.f90:456-592) with the HEVE short step:
    the volume-weighted totals of DENS and RHOT are conserved to round-off."""
    g = helpers.small_grid(10, 8, 14, stretched=True, halo=helpers.halo_of(scheme))
    c = mkinit.make_case("conserve heve", g, scheme, scheme, dt=0.5)
    k, i, j = np.meshgrid(np.arange(1, g.KA + 1), np.arange(1, g.IA + 1), np.arange(1, g.JA + 1), indexing="ij")
    st = c.state
    st["MOMZ"][...] = (k + i + j) * 0.01
    st["MOMX"][...] = (k * 2 + i + j) * 0.01
    st["MOMY"][...] = (k + i * 2 + j) * 0.01
    st["DENS"][...] = c.ref["REF_dens"] + (k * 2 + i * 2 + j) * 1e-4
    st["RHOT"][...] = st["DENS"] * (300.0 + (k + i + j * 2) * 0.01)
    for n in STATE:
        mkinit.periodic_fill(st[n], g)
    mkinit.vertical_fill(st, g)
    m0 = oracle.domain_sum(g, st["DENS"])
    t0 = oracle.domain_sum(g, st["RHOT"])
    _heve_steps(c, 3)
    assert abs(oracle.domain_sum(g, st["DENS"]) - m0) / m0 < 1e-13
    assert abs(oracle.domain_sum(g, st["RHOT"]) - t0) / t0 < 1e-13


def _energy_numpy(g, st, CZ):
    """Dry-air energies per cell restated with numpy (the cell-centre velocities of
    ATMOS_DIAGNOSTIC_CARTESC_get_vel on flat terrain, TEMP of rhot2temp_pres)."""
    ks, ke, is_, ie, js, je = g.KS - 1, g.KE, g.IS - 1, g.IE, g.JS - 1, g.JE
    D, MZ, MX, MY, RT = (st[n] for n in ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT"))
    d = D[ks:ke, is_:ie, js:je]
    w = np.empty_like(d)
    w[0] = MZ[ks, is_:ie, js:je] * 0.5
    w[1:-1] = 0.5 * (MZ[ks:ke - 2, is_:ie, js:je] + MZ[ks + 1:ke - 1, is_:ie, js:je]) / d[1:-1]
    w[-1] = 0.5 * MZ[ke - 2, is_:ie, js:je] / d[-1]
    u = 0.5 * (MX[ks:ke, is_ - 1:ie - 1, js:je] + MX[ks:ke, is_:ie, js:je]) / d
    v = 0.5 * (MY[ks:ke, is_:ie, js - 1:je - 1] + MY[ks:ke, is_:ie, js:je]) / d
    Rd, Cp = 287.04, 1004.64
    Cv = Cp - Rd
    pres = 100000.0 * (RT[ks:ke, is_:ie, js:je] * Rd / 100000.0) ** (Cp / Cv)
    temp = pres / (d * Rd)
    vol = g.CDZ[ks:ke, None, None] * g.CDX[None, is_:ie, None] * g.CDY[None, None, js:je]
    engp = d * 9.80665 * CZ[ks:ke, None, None]
    engk = 0.5 * d * (w * w + u * u + v * v)
    engi = d * temp * Cv
    return {n: float(np.sum(e * vol)) for n, e in
            (("ENGT", engp + engk + engi), ("ENGP", engp), ("ENGK", engk), ("ENGI", engi))}


def test_energy_budget_matches_a_direct_restatement():
    g = helpers.small_grid(IMAX=10, JMAX=8, KMAX=12, stretched=True)
    c = helpers.small_case(g, "CD4")
    helpers.perturb_state(c)
    got = oracle.energy_sum(g, c.state, g.CZ)
    want = _energy_numpy(g, c.state, g.CZ)
    for n in want:
        assert abs(got[n] - want[n]) <= 1e-12 * abs(want["ENGT"]), (n, got[n], want[n])
    assert abs(got["ENGT"] - (got["ENGP"] + got["ENGK"] + got["ENGI"])) <= 1e-12 * got["ENGT"]
    assert got["ENGK"] > 0.0 and got["ENGP"] > 0.0 and got["ENGI"] > 0.0


def test_energy_budget_of_a_state_at_rest_has_no_kinetic_part():
    g = helpers.small_grid(IMAX=6, JMAX=5, KMAX=10)
    c = helpers.small_case(g, "UD3", wind=0.0)
    st = {n: v.copy(order="F") for n, v in c.state.items()}
    for n in ("MOMZ", "MOMX", "MOMY"):
        st[n][...] = 0.0
    e = oracle.energy_sum(g, st, g.CZ)
    assert e["ENGK"] == 0.0
    assert e["ENGT"] == e["ENGP"] + e["ENGI"] or abs(e["ENGT"] - e["ENGP"] - e["ENGI"]) <= 1e-13 * e["ENGT"]
