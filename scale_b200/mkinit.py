"""Synthetic initial and reference states for the HEVI benchmarks and tests.

This is the preprocessing side of the workflow (scale-rm's mkinit), needed
only to produce inputs; it is not on the time-stepping path. It restates:

* the vertical and horizontal grid spacings of ATMOS_GRID_CARTESC_generate
  (scalelib/src/atmosphere/grid/scale_atmos_grid_cartesC.F90:694-841);
* a stratified base state theta(z) = theta_sfc * exp(N**2/g * z) as in
  MKINIT_gravitywave (scale-rm/src/preprocess/mod_mkinit.F90:1827) in
  hydrostatic balance by the Newton iteration of
  ATMOS_HYDROSTATIC_buildrho_atmos_0D/_1D
  (scalelib/src/atmosphere/common/scale_atmos_hydrostatic.F90:156-259,485-694);
* the reference pressure at the vertical halo levels of ATMOS_REFSTATE
  (scale_atmos_refstate.F90:831-834);
* cosine-squared warm bubbles with periodic distance (mod_mkinit.F90:560-607);
* the large-step preparation RT2P / DPRES0 / REF_rhot
  (scale_atmos_dyn_tstep_large_fvm_heve.F90:428-470), for short-step-only runs.

Noise comes from numpy's PCG64 generator with a fixed seed, so the oracle and
the GPU runs see bit-identical inputs.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

GRAV = 9.80665
RDRY = 287.04
CPDRY = 1004.64
CVDRY = CPDRY - RDRY
PRE00 = 100000.0
RVAP = 461.50
CPVAP = 1846.00
CVVAP = CPVAP - RVAP
CL = 4218.0
EPS = float(np.finfo(np.float64).eps)
HALO = 2
WIDE_SCHEMES = ("UD5", "CD6")  # 6-point flux schemes: IHALO = JHALO = 3


def halo_for(*schemes) -> int:
    """The lateral halo the flux schemes need (scale_atmos_dyn_fvm_flux.F90:742-749)."""
    return 3 if any(s in WIDE_SCHEMES for s in schemes) else HALO


@dataclass
class Grid:
    """Index set and 1-D spacings, 1-based reference arrays stored 0-based."""

    IMAX: int
    JMAX: int
    KMAX: int
    DX: float
    DY: float
    FZ: np.ndarray  # face heights of the interior levels KS..KE (KMAX values)
    halo: int = HALO  # IHALO = JHALO (3 for the UD5/CD6 flux schemes); KHALO is always 2

    def __post_init__(self):
        H = self.halo
        self.KA, self.IA, self.JA = self.KMAX + 2 * HALO, self.IMAX + 2 * H, self.JMAX + 2 * H
        self.KS, self.KE = 1 + HALO, self.KMAX + HALO
        self.IS, self.IE = 1 + H, self.IMAX + H
        self.JS, self.JE = 1 + H, self.JMAX + H
        KA, KS, KE = self.KA, self.KS, self.KE
        fz = np.zeros(KA + 1)  # FZ(0:KA)
        fz[KS - 1] = 0.0
        dz0 = self.FZ[0]
        for k in range(KS - 2, -1, -1):
            fz[k] = fz[k + 1] - dz0
        fz[KS : KE + 1] = self.FZ
        dzt = self.FZ[-1] - self.FZ[-2]
        for k in range(KE + 1, KA + 1):
            fz[k] = fz[k - 1] + dzt
        self.FZ_full = fz
        self.CZ = np.array([0.5 * (fz[k] + fz[k - 1]) for k in range(1, KA + 1)])
        self.CDZ = np.array([fz[k] - fz[k - 1] for k in range(1, KA + 1)])
        self.RCDZ = 1.0 / self.CDZ
        self.FDZ = np.array([self.CZ[k] - self.CZ[k - 1] for k in range(1, KA)])
        self.RFDZ = 1.0 / self.FDZ
        self.CDX = np.full(self.IA, float(self.DX))
        self.FDX = np.full(self.IA - 1, float(self.DX))
        self.RCDX = 1.0 / self.CDX
        self.RFDX = 1.0 / self.FDX
        self.CDY = np.full(self.JA, float(self.DY))
        self.FDY = np.full(self.JA - 1, float(self.DY))
        self.RCDY = 1.0 / self.CDY
        self.RFDY = 1.0 / self.FDY
        self.CX = (np.arange(1, self.IA + 1) - self.IS + 0.5) * self.DX
        self.CY = (np.arange(1, self.JA + 1) - self.JS + 0.5) * self.DY

    @property
    def shape(self):
        """numpy shape of a (KA,IA,JA) field in Fortran order."""
        return (self.KA, self.IA, self.JA)

    @property
    def cells(self) -> int:
        return self.IMAX * self.JMAX * self.KMAX

    def zeros(self, *extra):
        return np.zeros(self.shape + tuple(extra), dtype=np.float64, order="F")

    def index_dict(self):
        return dict(KA=self.KA, IA=self.IA, JA=self.JA, KS=self.KS, KE=self.KE, IS=self.IS, IE=self.IE,
                    JS=self.JS, JE=self.JE, KMAX=self.KMAX, IMAX=self.IMAX, JMAX=self.JMAX,
                    KHALO=HALO, IHALO=self.halo, JHALO=self.halo, IBLOCK=self.IMAX, JBLOCK=self.JMAX)


def uniform_grid(IMAX, JMAX, KMAX, DX, DY, DZ, halo=HALO) -> Grid:
    return Grid(IMAX, JMAX, KMAX, DX, DY, DZ * np.arange(1, KMAX + 1, dtype=np.float64), halo)


def stretched_grid(IMAX, JMAX, KMAX, DX, DY, dz_bottom, dz_top, halo=HALO) -> Grid:
    """Face heights whose spacing grows geometrically from dz_bottom to dz_top."""
    r = (dz_top / dz_bottom) ** (1.0 / (KMAX - 1))
    dz = dz_bottom * r ** np.arange(KMAX)
    return Grid(IMAX, JMAX, KMAX, DX, DY, np.cumsum(dz), halo)


# ---------------------------------------------------------------------------
# hydrostatic base state
# ---------------------------------------------------------------------------
def _newton_layer(pott2, R2, CPovCV2, dens1, pres1, dz):
    """buildrho Newton iteration for one layer (scale_atmos_hydrostatic.F90:537-575)."""
    criteria = np.sqrt(EPS)
    dens_s, dens2 = 0.0, dens1
    for _ in range(100):
        if abs(dens2 - dens_s) <= criteria:
            break
        dens_s = dens2
        pres2 = PRE00 * (dens_s * R2 * pott2 / PRE00) ** CPovCV2
        dhyd = (pres1 - pres2) / dz - GRAV * 0.5 * (dens1 + dens_s)
        dgrd = -pres2 * CPovCV2 / dens_s / dz - GRAV * 0.5
        dens2 = dens_s - dhyd / dgrd
    else:
        raise RuntimeError("hydrostatic iteration did not converge")
    pres2 = PRE00 * (dens2 * R2 * pott2 / PRE00) ** CPovCV2
    return dens2, pres2


def base_state(g: Grid, theta_sfc=300.0, bvf=0.01, pres_sfc=1.0e5, qv=None):
    """Stratified hydrostatic column: returns dict of 1-D (KA) arrays."""
    KA, KS, KE = g.KA, g.KS, g.KE
    pott = theta_sfc * np.exp(bvf * bvf / GRAV * g.CZ)
    qv = np.zeros(KA) if qv is None else qv
    Rtot = RDRY * (1.0 - qv) + RVAP * qv
    CVtot = CVDRY * (1.0 - qv) + CVVAP * qv
    CPtot = CPDRY * (1.0 - qv) + CPVAP * qv
    CPovCV = CPtot / CVtot
    dens = np.zeros(KA)
    pres = np.zeros(KA)
    dens_sfc = PRE00 / RDRY / theta_sfc * (pres_sfc / PRE00) ** (CVDRY / CPDRY)
    pres_sfc_ = PRE00 * (dens_sfc * RDRY * theta_sfc / PRE00) ** (CPDRY / CVDRY)
    dens[KS - 1], pres[KS - 1] = _newton_layer(pott[KS - 1], Rtot[KS - 1], CPovCV[KS - 1], dens_sfc, pres_sfc_,
                                               g.CZ[KS - 1] - g.FZ_full[KS - 1])
    for k in range(KS + 1, KE + 1):
        dens[k - 1], pres[k - 1] = _newton_layer(pott[k - 1], Rtot[k - 1], CPovCV[k - 1], dens[k - 2], pres[k - 2],
                                                 g.CZ[k - 1] - g.CZ[k - 2])
    dens[: KS - 1] = dens[KS - 1]
    dens[KE:] = dens[KE - 1]
    temp = pres / (np.where(dens > 0, dens, 1.0) * Rtot)
    phi = GRAV * g.CZ
    # halo pressure extrapolation of the reference state (refstate.F90:831-834)
    pres[KS - 2] = pres[KS] - dens[KS - 1] * (phi[KS - 2] - phi[KS])
    pres[KE] = pres[KE - 2] - dens[KE - 1] * (phi[KE] - phi[KE - 2])
    pres[: KS - 2] = pres[KS - 2]
    pres[KE + 1 :] = pres[KE]
    return dict(dens=dens, pres=pres, pott=pott, temp=temp, phi=phi)


def _bcast(col, g: Grid):
    return np.asfortranarray(np.broadcast_to(col[:, None, None], g.shape).copy())


def bubble(g: Grid, cx, cy, cz, rx, ry, rz):
    """cos**2 bubble with periodic x/y distance (mod_mkinit.F90:580-601)."""
    Lx = g.IMAX * g.DX
    Ly = g.JMAX * g.DY
    dz = ((g.CZ - cz) / rz) ** 2
    dx = np.minimum(np.minimum(((g.CX - cx) / rx) ** 2, ((g.CX - cx - Lx) / rx) ** 2), ((g.CX - cx + Lx) / rx) ** 2)
    dy = np.minimum(np.minimum(((g.CY - cy) / ry) ** 2, ((g.CY - cy - Ly) / ry) ** 2), ((g.CY - cy + Ly) / ry) ** 2)
    dist = dz[:, None, None] + dx[None, :, None] + dy[None, None, :]
    return np.asfortranarray(np.cos(0.5 * np.pi * np.sqrt(np.minimum(dist, 1.0))) ** 2)


def add_bubble(theta: np.ndarray, g: Grid, cx, cy, cz, rx, ry, rz, amp) -> np.ndarray:
    """theta + amp * bubble(...), evaluated only on the bubble's support.

    Outside the support the cos**2 term is cos(pi/2)**2, about 4e-33, which
    leaves a potential temperature of a few hundred K unchanged in FP64; so
    the result equals the full-domain sum bit for bit (checked by the tests),
    at a fraction of the cost on large domains."""
    Lx = g.IMAX * g.DX
    Ly = g.JMAX * g.DY
    dz = ((g.CZ - cz) / rz) ** 2
    dx = np.minimum(np.minimum(((g.CX - cx) / rx) ** 2, ((g.CX - cx - Lx) / rx) ** 2), ((g.CX - cx + Lx) / rx) ** 2)
    dy = np.minimum(np.minimum(((g.CY - cy) / ry) ** 2, ((g.CY - cy - Ly) / ry) ** 2), ((g.CY - cy + Ly) / ry) ** 2)
    kk, ii, jj = np.nonzero(dz < 1.0)[0], np.nonzero(dx < 1.0)[0], np.nonzero(dy < 1.0)[0]
    if len(kk) == 0 or len(ii) == 0 or len(jj) == 0:
        return theta
    dist = dz[kk][:, None, None] + dx[ii][None, :, None] + dy[jj][None, None, :]
    sel = np.ix_(kk, ii, jj)
    theta[sel] = theta[sel] + amp * np.cos(0.5 * np.pi * np.sqrt(np.minimum(dist, 1.0))) ** 2
    return theta


def periodic_fill(a: np.ndarray, g: Grid):
    """Periodic lateral halo of one (KA,IA,JA) field (all k)."""
    I, J = g.IMAX, g.JMAX
    a[:, : g.IS - 1, :] = a[:, g.IE - (g.IS - 1) : g.IE, :]
    a[:, g.IE :, :] = a[:, g.IS - 1 : g.IS - 1 + (g.IA - g.IE), :]
    a[:, :, : g.JS - 1] = a[:, :, g.JE - (g.JS - 1) : g.JE]
    a[:, :, g.JE :] = a[:, :, g.JS - 1 : g.JS - 1 + (g.JA - g.JE)]
    del I, J
    return a


def vertical_fill(st: dict, g: Grid):
    """Vertical boundary values as after each short step (tstep_large:910-926)."""
    KS, KE = g.KS, g.KE
    for n in ("DENS", "MOMX", "MOMY", "RHOT"):
        a = st[n]
        a[: KS - 1] = a[KS - 1]
        a[KE:] = a[KE - 1]
    st["MOMZ"][: KS - 1] = 0.0
    st["MOMZ"][KE - 1 :] = 0.0


# ---------------------------------------------------------------------------
# tracers
# ---------------------------------------------------------------------------
TRACER_NAMES = ("QV", "QC", "QR")
# (R, CV, CP, MASS) per tracer, as registered by the Kessler-type hydrometeor set
TRACER_PROPS = {"QV": (RVAP, CVVAP, CPVAP, 1.0), "QC": (0.0, CL, CL, 1.0), "QR": (0.0, CL, CL, 1.0)}


def qsat_water(temp, pres):
    """Saturation mixing ratio over water (Tetens formula), used only to set the initial QV."""
    es = 611.2 * np.exp(17.67 * (temp - 273.15) / (temp - 29.65))
    return 0.622 * es / np.maximum(pres - 0.378 * es, 1.0)


@dataclass
class Case:
    name: str
    g: Grid
    scheme: str
    scheme_tracer: str
    dt: float
    dtl: float
    nd_coef: float = 1.0e-4
    state: dict = field(default_factory=dict)   # DENS MOMZ MOMX MOMY RHOT (+ QTRC)
    ref: dict = field(default_factory=dict)     # REF_dens REF_pott REF_pres PHI
    QA: int = 0
    fct: bool = False


def make_case(name: str, g: Grid, scheme="UD3", scheme_tracer="UD3", dt=1.0, dtl=5.0, bubbles=(), theta_noise=0.0,
              noise_kind="uniform", wind_noise=0.0, noise_top=1.0e30, tracers=0, fct=False, seed=0, u0=0.0, v0=0.0,
              rh0=0.8, rh_scale=3000.0) -> Case:
    rng = np.random.Generator(np.random.PCG64(seed))
    base = base_state(g)
    DENS = _bcast(base["dens"], g)
    theta = _bcast(base["pott"], g)
    for (cx, cy, cz, rx, ry, rz, amp) in bubbles:
        theta = add_bubble(theta, g, cx, cy, cz, rx, ry, rz, amp)
    shp = g.shape
    low = (g.CZ <= noise_top)[:, None, None]
    if theta_noise > 0.0:
        if noise_kind == "uniform":
            n = rng.uniform(-theta_noise, theta_noise, size=shp)
        else:
            n = rng.normal(0.0, theta_noise, size=shp)
        theta = theta + np.where(low, n, 0.0)
    MOMX = DENS * u0
    MOMY = DENS * v0
    if wind_noise > 0.0:
        MOMX = MOMX + DENS * np.where(low, rng.normal(0.0, wind_noise, size=shp), 0.0)
        MOMY = MOMY + DENS * np.where(low, rng.normal(0.0, wind_noise, size=shp), 0.0)
    st = {
        "DENS": np.asfortranarray(DENS),
        "MOMZ": g.zeros(),
        "MOMX": np.asfortranarray(MOMX),
        "MOMY": np.asfortranarray(MOMY),
        "RHOT": np.asfortranarray(DENS * theta),
    }
    for n in st:
        periodic_fill(st[n], g)
    vertical_fill(st, g)
    ref = {
        "REF_dens": _bcast(base["dens"], g),
        "REF_pott": _bcast(base["pott"], g),
        "REF_pres": _bcast(base["pres"], g),
        "PHI": _bcast(base["phi"], g),
    }
    c = Case(name, g, scheme, scheme_tracer, dt, dtl, state=st, ref=ref, QA=tracers, fct=fct)
    if tracers:
        q = g.zeros(tracers)
        rh = rh0 * np.exp(-g.CZ / rh_scale)
        qv = rh * qsat_water(base["temp"], np.maximum(base["pres"], 1.0))
        q[..., 0] = np.asfortranarray(np.broadcast_to(qv[:, None, None], shp))
        q[: g.KS - 1] = 0.0
        q[g.KE :] = 0.0
        st["QTRC"] = q
    return c


def aq_props(QA: int):
    names = TRACER_NAMES[:QA]
    arr = np.array([TRACER_PROPS[n] for n in names], dtype=np.float64).reshape(QA, 4)
    return [np.ascontiguousarray(arr[:, c]) for c in range(4)]


def large_prep(case: Case):
    """RT2P, DPRES0 and REF_rhot of tstep_large_fvm_heve.F90:428-470 (numpy, moist form)."""
    g = case.g
    st, ref = case.state, case.ref
    KS, KE = g.KS, g.KE
    RT2P = g.zeros()
    DPRES0 = g.zeros()
    REF_rhot = g.zeros()
    sl = slice(KS - 1, KE)
    Rtot = np.zeros(st["RHOT"][sl].shape)
    CVtot = np.zeros_like(Rtot)
    CPtot = np.zeros_like(Rtot)
    QDRY = np.ones_like(Rtot)
    if case.QA:
        R, CV, CP, M = aq_props(case.QA)
        for iq in range(case.QA):
            q = st["QTRC"][sl, :, :, iq]
            Rtot = Rtot + R[iq] * q
            CVtot = CVtot + CV[iq] * q
            CPtot = CPtot + CP[iq] * q
            QDRY = QDRY - q * M[iq]
    Rtot = Rtot + RDRY * QDRY
    CVtot = CVtot + CVDRY * QDRY
    CPtot = CPtot + CPDRY * QDRY
    rhot = st["RHOT"][sl]
    PRES = PRE00 * (Rtot * rhot / PRE00) ** (CPtot / CVtot)
    RT2P[sl] = CPtot / CVtot * PRES / rhot
    DPRES0[sl] = PRES - ref["REF_pres"][sl]
    REF_rhot[sl] = rhot
    DPRES0[KS - 2] = DPRES0[KS] + (ref["REF_pres"][KS] - ref["REF_pres"][KS - 2])
    DPRES0[KE] = DPRES0[KE - 2] + (ref["REF_pres"][KE - 2] - ref["REF_pres"][KE])
    return RT2P, DPRES0, REF_rhot


# ---------------------------------------------------------------------------
# the benchmark configurations
# ---------------------------------------------------------------------------
def config(n: int, scale: float = 1.0, seed: int = 0) -> Case:
    """Synthetic stand-ins for the five published configurations.

    scale < 1 shrinks the horizontal domain (for tests); the vertical grid and
    physics settings are kept.
    """
    def h(nn):
        return max(8, int(round(nn * scale)))

    if n == 1:
        g = uniform_grid(h(40), h(40), 80, 500.0, 500.0, 250.0)
        Lx, Ly = g.IMAX * 500.0, g.JMAX * 500.0
        return make_case("warm bubble 40x40x80 UD3", g, "UD3", "UD3", dt=1.0, dtl=5.0,
                         bubbles=[(min(10000.0, Lx / 2), min(10000.0, Ly / 2), 2000.0, 4000.0, 4000.0, 4000.0, 3.0)],
                         theta_noise=0.01, noise_kind="uniform", seed=seed)
    if n == 2:
        g = stretched_grid(h(512), h(512), 128, 250.0, 250.0, 50.0, 400.0)
        return make_case("stretched 512x512x128 CD4, 3 tracers FCT", g, "CD4", "UD3", dt=0.5, dtl=2.5,
                         theta_noise=0.1, noise_kind="normal", wind_noise=0.5, noise_top=1000.0,
                         tracers=3, fct=True, seed=seed)
    if n == 4:
        g = uniform_grid(h(1024), h(1024), 96, 200.0, 200.0, 200.0)
        rng = np.random.Generator(np.random.PCG64(seed + 4))
        Lx, Ly = g.IMAX * 200.0, g.JMAX * 200.0
        bub = [(rng.uniform(0, Lx), rng.uniform(0, Ly), rng.uniform(1000.0, 4000.0), 2000.0, 2000.0, 1500.0,
                rng.uniform(1.0, 3.0)) for _ in range(32)]
        # dt = 0.4 s keeps the horizontal acoustic Courant number of the 500 m /
        # 1 s tutorial (about 0.7); 1 s at 200 m would exceed the explicit limit
        return make_case("multi-bubble 1024x1024x96", g, "UD3", "UD3", dt=0.4, dtl=2.0, bubbles=bub, seed=seed)
    if n == 5:
        g = uniform_grid(h(128), h(128), 64, 500.0, 500.0, 500.0)
        Lx, Ly = g.IMAX * 500.0, g.JMAX * 500.0
        return make_case("warm bubble 128x128x64", g, "UD3", "UD3", dt=1.0, dtl=5.0,
                         bubbles=[(Lx / 2, Ly / 2, 2000.0, 4000.0, 4000.0, 4000.0, 3.0)],
                         theta_noise=0.01, seed=seed)
    raise ValueError(f"unknown configuration {n}")


# ---------------------------------------------------------------------------
# the uneven ensemble
# ---------------------------------------------------------------------------
# 48 members of three sizes (IMAX, JMAX, KMAX), all at dx = dy = 500 m with
# the tutorial's 250 m levels
ENSEMBLE_SIZES = [(64, 64, 64)] * 16 + [(128, 128, 96)] * 16 + [(256, 256, 96)] * 16


def ensemble_member(IMAX: int, JMAX: int, KMAX: int, m: int, seed: int = 0, scheme: str = "UD3") -> Case:
    """Member m: one warm bubble at a seeded position with a seeded amplitude
    in [1, 4] K, and its own seeded +-0.01 K theta noise."""
    g = uniform_grid(IMAX, JMAX, KMAX, 500.0, 500.0, 250.0, halo=halo_for(scheme))
    rng = np.random.Generator(np.random.PCG64(seed + 3000 + m))
    Lx, Ly = g.IMAX * 500.0, g.JMAX * 500.0
    bub = [(rng.uniform(0.0, Lx), rng.uniform(0.0, Ly), 2000.0, 4000.0, 4000.0, 4000.0, rng.uniform(1.0, 4.0))]
    return make_case(f"ensemble member {m} {IMAX}x{JMAX}x{KMAX}", g, scheme, scheme, dt=1.0, dtl=5.0, bubbles=bub,
                     theta_noise=0.01, noise_kind="uniform", seed=seed + 100 + m)


def ensemble(scale: float = 1.0, seed: int = 0, sizes=None, scheme: str = "UD3") -> list[Case]:
    """The members of the uneven ensemble (scale < 1 shrinks the horizontal
    sizes, for tests; sizes replaces the member list)."""
    sizes = ENSEMBLE_SIZES if sizes is None else sizes
    return [ensemble_member(max(8, int(round(I * scale))), max(8, int(round(J * scale))), K, m, seed, scheme)
            for m, (I, J, K) in enumerate(sizes)]
