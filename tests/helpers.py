"""Input builders shared by the tests (seeded, identical for the oracle and the GPU)."""
from __future__ import annotations

import numpy as np

import oracle
from scale_b200 import mkinit


def small_grid(IMAX=12, JMAX=10, KMAX=16, DX=500.0, DY=400.0, DZ=250.0, stretched=False, halo=2):
    if stretched:
        return mkinit.stretched_grid(IMAX, JMAX, KMAX, DX, DY, 60.0, 400.0, halo=halo)
    return mkinit.uniform_grid(IMAX, JMAX, KMAX, DX, DY, DZ, halo=halo)


def halo_of(scheme):
    """IHALO = JHALO a flux scheme needs (scale_atmos_dyn_fvm_flux.F90:742-749 for UD5/CD6)."""
    return mkinit.halo_for(scheme)


def small_case(g, scheme="UD3", seed=1, tracers=0, wind=2.0):
    Lx, Ly = g.IMAX * g.DX, g.JMAX * g.DY
    c = mkinit.make_case("test", g, scheme, scheme, dt=1.0, dtl=5.0,
                         bubbles=[(Lx * 0.4, Ly * 0.6, 1500.0, Lx * 0.3, Ly * 0.3, 1500.0, 3.0)],
                         theta_noise=0.05, noise_kind="normal", wind_noise=wind, seed=seed, tracers=tracers,
                         u0=3.0, v0=-2.0)
    return c


def perturb_state(c, seed=7, w_amp=0.5):
    """Random vertical momentum (both signs, so every upwind branch is taken)."""
    g, st = c.g, c.state
    rng = np.random.Generator(np.random.PCG64(seed))
    st["MOMZ"][...] = st["DENS"] * rng.normal(0.0, w_amp, size=g.shape)
    mkinit.periodic_fill(st["MOMZ"], g)
    mkinit.vertical_fill(st, g)


def short_inputs(c, dtrk=0.5, seed=3, full=True):
    """Every input of one HEVI stage, reference names. full=True turns on the
    optional terms (tendencies, Coriolis, Rayleigh and divergence damping)."""
    g, st, ref = c.g, c.state, c.ref
    rng = np.random.Generator(np.random.PCG64(seed))
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    nd = g.zeros(5, 3)
    oracle.numfilter(g, nd, st, ref, DT=1.0, ND_COEF=1e-3 if full else 1e-4)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    a = dict(
        DENS0=st["DENS"].copy(order="F"), MOMZ0=st["MOMZ"].copy(order="F"), MOMX0=st["MOMX"].copy(order="F"),
        MOMY0=st["MOMY"].copy(order="F"), RHOT0=st["RHOT"].copy(order="F"),
        DPRES0=DPRES0, RT2P=RT2P, REF_dens=ref["REF_dens"], REF_rhot=REF_rhot, PHI=ref["PHI"],
        num_diff=nd, CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY,
        RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY, GSQRT=GS, J13G=J13, J23G=J23, J33G=1.0, MAPF=MAPF, dtrk=dtrk,
    )
    # the stage input differs from the stage-0 state, as in RK stages 2-4
    for n, amp in (("DENS", 1e-4), ("MOMZ", 1e-2), ("MOMX", 1e-2), ("MOMY", 1e-2), ("RHOT", 1e-2)):
        x = st[n] + amp * rng.normal(size=g.shape)
        if n == "MOMZ":
            x[: g.KS - 1] = 0.0
            x[g.KE - 1 :] = 0.0
        mkinit.periodic_fill(x, g)
        a[n] = np.asfortranarray(x)
    for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t"):
        a[n] = np.asfortranarray(1e-5 * rng.normal(size=g.shape)) if full else g.zeros()
    a["CORIOLI"] = np.asfortranarray(np.full((g.IA, g.JA), 1.0e-4 if full else 0.0)
                                     + (1e-6 * rng.normal(size=(g.IA, g.JA)) if full else 0.0))
    wd = np.zeros(g.KA)
    if full:
        wd[g.KE - 4 : g.KE] = np.linspace(0.001, 0.01, 4)
    a["wdamp_coef"] = wd
    a["divdmp_coef"] = 0.1 if full else 0.0
    if full:
        ddiv = g.zeros()
        oracle.divergence(g, ddiv, a, GS, J13, J23, 1.0, MAPF)
        a["DDIV"] = ddiv
    else:
        a["DDIV"] = g.zeros()
    return a


def stage_outputs(g, fill=np.nan):
    """Output arrays pre-filled with a sentinel so unwritten cells are visible."""
    o = {n: np.full(g.shape, fill, order="F") for n in ("DENS_RK", "MOMZ_RK", "MOMX_RK", "MOMY_RK", "RHOT_RK")}
    o["mflx_hi"] = np.full(g.shape + (3,), fill, order="F")
    o["tflx_hi"] = np.full(g.shape + (3,), fill, order="F")
    return o


def same(a: np.ndarray, b: np.ndarray) -> bool:
    """Bit-level equality that treats NaN sentinels in the same place as equal and +0 == -0."""
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def max_rel(a: np.ndarray, b: np.ndarray) -> float:
    m = np.isfinite(a) & np.isfinite(b)
    den = np.maximum(np.abs(b[m]), 1e-300)
    return float(np.max(np.abs(a[m] - b[m]) / np.maximum(den, np.max(np.abs(b[m])) * 1e-12))) if m.any() else 0.0
