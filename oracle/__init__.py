"""ctypes binding of the CPU oracle (oracle/build/liboracle.so).

Test infrastructure: the FP64 C restatement of the reference routines that the
CUDA product path is checked against. Only tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py use it. See scale_oracle.h for the
restatement's scope and pinning status ("parity unpinned" against the Fortran
build: no Fortran compiler or golden vectors exist for this path).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "build" / "liboracle.so"
UD3, CD4, KOREN, CD2, UD5, CD6 = 1, 2, 3, 4, 5, 6
SCHEMES = {"UD3": UD3, "CD4": CD4, "UD3KOREN1993": KOREN, "CD2": CD2, "UD5": UD5, "CD6": CD6}
WIDE = ("UD5", "CD6")  # 6-point schemes: IHALO = JHALO = 3


class Dims(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("KA", "IA", "JA", "KS", "KE", "IS", "IE", "JS", "JE", "KMAX", "IMAX", "JMAX",
                                       "IHALO", "JHALO", "IEH", "JEH")]


_lib = None

def _signatures() -> dict[str, str]:
    """Argument kinds of every og_* prototype in scale_oracle.h:
    D = const og_dims*, d = double*, s = double, i = int."""
    import re

    text = (HERE / "scale_oracle.h").read_text()
    out = {}
    for m in re.finditer(r"\n(?:int|void|double)\s+(og_\w+)\(([^;]*?)\);", text):
        kinds = []
        for p in m.group(2).split(","):
            p = " ".join(p.split())
            if not p or p == "void":
                continue
            if "og_dims" in p:
                kinds.append("D")
            elif "*" in p:
                kinds.append("d")
            elif p.startswith("double"):
                kinds.append("s")
            else:
                kinds.append("i")
        out[m.group(1)] = " ".join(kinds)
    return out


_RESTYPE = {"og_halo_periodic": None, "og_divergence": None, "og_hevi_max_residual": C.c_double,
            "og_domain_sum": C.c_double, "og_short_type": None, "og_tinteg_short_type": None,
            "og_energy_sum": None}


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        raise FileNotFoundError(f"{LIB} is missing: run `make -C oracle` (or __graft_entry__.build())")
    lib = C.CDLL(str(LIB))
    kinds = {"D": C.POINTER(Dims), "d": C.c_void_p, "s": C.c_double, "i": C.c_int}
    for name, sig in _signatures().items():
        f = getattr(lib, name)
        f.argtypes = [kinds[k] for k in sig.split()]
        f.restype = _RESTYPE.get(name, C.c_int)
    lib.og_set_halo_exchange.argtypes = [HALO_FN, C.c_void_p]
    lib.og_set_halo_exchange.restype = None
    _lib = lib
    return lib


def dims(g) -> Dims:
    return Dims(KA=g.KA, IA=g.IA, JA=g.JA, KS=g.KS, KE=g.KE, IS=g.IS, IE=g.IE, JS=g.JS, JE=g.JE, KMAX=g.KMAX,
                IMAX=g.IMAX, JMAX=g.JMAX, IHALO=g.IS - 1, JHALO=g.JS - 1, IEH=g.IE, JEH=g.JE)


def _p(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "bad array"
    return a.ctypes.data


def _call(name, g, *args):
    lib = load()
    d = dims(g)
    conv = [C.byref(d)]
    for a in args:
        conv.append(_p(a) if (a is None or isinstance(a, np.ndarray)) else a)
    rc = getattr(lib, name)(*conv)
    if _RESTYPE.get(name, C.c_int) is C.c_int and rc != 0:
        raise RuntimeError(f"{name} failed with status {rc}")
    return rc


def num_threads() -> int:
    return load().og_num_threads()


def flat_metrics(g):
    """GSQRT = 1, J13G = J23G = 0 (KA,IA,JA,7) and MAPF = 1 (IA,JA,2,4)."""
    GS = np.ones(g.shape + (7,), order="F")
    J = np.zeros(g.shape + (7,), order="F")
    M = np.ones((g.IA, g.JA, 2, 4), order="F")
    return GS, J, J.copy(order="F"), M


def tstep_short(g, scheme, o, a):
    """One HEVI stage: o holds output arrays, a the inputs (reference names)."""
    return _call("og_tstep_short_fvm_hevi", g, SCHEMES[scheme],
                 o["DENS_RK"], o["MOMZ_RK"], o["MOMX_RK"], o["MOMY_RK"], o["RHOT_RK"], o["mflx_hi"], o["tflx_hi"],
                 a["DENS0"], a["MOMZ0"], a["MOMX0"], a["MOMY0"], a["RHOT0"],
                 a["DENS"], a["MOMZ"], a["MOMX"], a["MOMY"], a["RHOT"],
                 a["DENS_t"], a["MOMZ_t"], a["MOMX_t"], a["MOMY_t"], a["RHOT_t"],
                 a["DPRES0"], a["RT2P"], a["CORIOLI"], a["num_diff"], a["wdamp_coef"], float(a["divdmp_coef"]), a["DDIV"],
                 a["CDZ"], a["FDZ"], a["FDX"], a["FDY"], a["RCDZ"], a["RCDX"], a["RCDY"], a["RFDZ"], a["RFDX"], a["RFDY"],
                 a["PHI"], a["GSQRT"], a["J13G"], a["J23G"], float(a["J33G"]), a["MAPF"], a["REF_dens"], a["REF_rhot"],
                 float(a["dtrk"]))


def tstep_short_heve(g, scheme, o, a):
    """One HEVE stage (fully explicit), same arguments as tstep_short."""
    return _call("og_tstep_short_fvm_heve", g, SCHEMES[scheme],
                 o["DENS_RK"], o["MOMZ_RK"], o["MOMX_RK"], o["MOMY_RK"], o["RHOT_RK"], o["mflx_hi"], o["tflx_hi"],
                 a["DENS0"], a["MOMZ0"], a["MOMX0"], a["MOMY0"], a["RHOT0"],
                 a["DENS"], a["MOMZ"], a["MOMX"], a["MOMY"], a["RHOT"],
                 a["DENS_t"], a["MOMZ_t"], a["MOMX_t"], a["MOMY_t"], a["RHOT_t"],
                 a["DPRES0"], a["RT2P"], a["CORIOLI"], a["num_diff"], a["wdamp_coef"], float(a["divdmp_coef"]), a["DDIV"],
                 a["CDZ"], a["FDZ"], a["FDX"], a["FDY"], a["RCDZ"], a["RCDX"], a["RCDY"], a["RFDZ"], a["RFDX"], a["RFDY"],
                 a["PHI"], a["GSQRT"], a["J13G"], a["J23G"], float(a["J33G"]), a["MAPF"], a["REF_dens"], a["REF_rhot"],
                 float(a["dtrk"]))


def tinteg_short_rk4(g, scheme, x, a, short="HEVI"):
    """RK4 short step; x holds DENS..RHOT, mflx_hi, tflx_hi (updated in place).
    short selects the registered short step, "HEVI" or "HEVE"."""
    return _call({"HEVI": "og_tinteg_short_rk4", "HEVE": "og_tinteg_short_rk4_heve"}[short], g, SCHEMES[scheme],
                 x["DENS"], x["MOMZ"], x["MOMX"], x["MOMY"], x["RHOT"], x["mflx_hi"], x["tflx_hi"],
                 a["DENS_t"], a["MOMZ_t"], a["MOMX_t"], a["MOMY_t"], a["RHOT_t"],
                 a["DPRES0"], a["RT2P"], a["CORIOLI"], a["num_diff"], a["wdamp_coef"], float(a["divdmp_coef"]), a["DDIV"],
                 a["CDZ"], a["FDZ"], a["FDX"], a["FDY"], a["RCDZ"], a["RCDX"], a["RCDY"], a["RFDZ"], a["RFDX"], a["RFDY"],
                 a["PHI"], a["GSQRT"], a["J13G"], a["J23G"], float(a["J33G"]), a["MAPF"], a["REF_dens"], a["REF_rhot"],
                 float(a["dt"]))


def tinteg_short_rk3(g, scheme, x, a, ws2002=True, short="HEVI"):
    """RK3 short step (RK3WS2002 or, with ws2002=False, Heun's RK3) with the
    short step `short`; x as for tinteg_short_rk4."""
    load().og_short_type({"HEVI": 0, "HEVE": 1}[short])
    try:
        return _call("og_tinteg_short_rk3", g, SCHEMES[scheme], int(bool(ws2002)),
                     x["DENS"], x["MOMZ"], x["MOMX"], x["MOMY"], x["RHOT"], x["mflx_hi"], x["tflx_hi"],
                     a["DENS_t"], a["MOMZ_t"], a["MOMX_t"], a["MOMY_t"], a["RHOT_t"],
                     a["DPRES0"], a["RT2P"], a["CORIOLI"], a["num_diff"], a["wdamp_coef"], float(a["divdmp_coef"]),
                     a["DDIV"], a["CDZ"], a["FDZ"], a["FDX"], a["FDY"], a["RCDZ"], a["RCDX"], a["RCDY"], a["RFDZ"],
                     a["RFDX"], a["RFDY"], a["PHI"], a["GSQRT"], a["J13G"], a["J23G"], float(a["J33G"]), a["MAPF"],
                     a["REF_dens"], a["REF_rhot"], float(a["dt"]))
    finally:
        load().og_short_type(0)


def halo(g, var, nfields=1):
    _call("og_halo_periodic", g, var, int(nfields))


# int (*)(double *var, int nfields, void *user)
HALO_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int, C.c_void_p)
_halo_cb = None  # the registered callback, kept alive while set


def set_halo_exchange(g, fn) -> None:
    """While fn is set, every halo fill of the oracle calls fn(fields) with
    fields a list of the nfields (KA,IA,JA) arrays (1-D float64 views of the
    oracle's memory, in the grid g's Fortran order), to be filled in place;
    None restores the periodic fill (og_set_halo_exchange)."""
    global _halo_cb
    lib = load()
    if fn is None:
        lib.og_set_halo_exchange(HALO_FN(), None)
        _halo_cb = None
        return
    n3 = g.KA * g.IA * g.JA

    def tramp(var, nfields, user):
        flat = np.ctypeslib.as_array(var, shape=(nfields * n3,))
        fn([flat[q * n3:(q + 1) * n3] for q in range(nfields)])
        return 0

    _halo_cb = HALO_FN(tramp)
    lib.og_set_halo_exchange(_halo_cb, None)


def numfilter(g, num_diff, st, ref, DT, ND_COEF=1e-4, ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=1):
    return _call("og_numfilter_coef", g, num_diff, st["DENS"], st["MOMZ"], st["MOMX"], st["MOMY"], st["RHOT"],
                 g.CDZ, g.CDX, g.CDY, g.FDZ, g.FDX, g.FDY, float(DT), ref["REF_dens"], ref["REF_pott"],
                 float(ND_COEF), int(ND_ORDER), float(ND_SFC_FACT), int(ND_USE_RS))


def divergence(g, DDIV, st, GSQRT, J13G, J23G, J33G, MAPF):
    _call("og_divergence", g, DDIV, st["MOMZ"], st["MOMX"], st["MOMY"], GSQRT, J13G, J23G, float(J33G), MAPF,
          g.RCDZ, g.RCDX, g.RCDY, g.RFDZ, g.FDZ)


def tstep_tracer(g, scheme, QTRCo, QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff_q, GSQRT, MAPF_XY, dtl,
                 fct, along):
    return _call("og_tstep_tracer_fvm_heve", g, SCHEMES[scheme], QTRCo, QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi,
                 num_diff_q, GSQRT, MAPF_XY, g.CDZ, g.RCDZ, g.RCDX, g.RCDY, float(dtl), int(fct), int(along))


def tinteg_tracer_rk3(g, scheme, QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff_q, GSQRT, MAPF_XY, dtl,
                      fct, along):
    return _call("og_tinteg_tracer_rk3", g, SCHEMES[scheme], QTRC, QTRC0, RHOQ_t, DENS0, DENS, mflx_hi, num_diff_q,
                 GSQRT, MAPF_XY, g.CDZ, g.RCDZ, g.RCDX, g.RCDY, float(dtl), int(fct), int(along))


def tstep_large(g, scheme, scheme_tracer, st, out, tp, ref, aq, GSQRT, J13G, J23G, MAPF, CORIOLI, wdamp, dtl, dts,
                ND_COEF=1e-4, divdmp=0.0, fct=False, along=True, QA=0, ND_ORDER=1, short="HEVI", tinteg="RK4"):
    """Large step of the dynamics; st (DENS..RHOT, QTRC) is advanced in place.
    short is the registered short step ("HEVI" or "HEVE"), tinteg the short
    integrator ("RK4", "RK3" or "RK3WS2002")."""
    QTRC = st.get("QTRC") if QA else None
    R, CV, CP, M = aq if QA else (None, None, None, None)
    load().og_short_type({"HEVI": 0, "HEVE": 1}[short])
    load().og_tinteg_short_type({"RK4": 0, "RK3": 1, "RK3WS2002": 2}[tinteg])
    try:
        return _tstep_large(g, scheme, scheme_tracer, st, out, tp, ref, GSQRT, J13G, J23G, MAPF, CORIOLI, wdamp,
                            dtl, dts, ND_COEF, divdmp, fct, along, QA, ND_ORDER, QTRC, R, CV, CP, M)
    finally:
        load().og_short_type(0)
        load().og_tinteg_short_type(0)


def _tstep_large(g, scheme, scheme_tracer, st, out, tp, ref, GSQRT, J13G, J23G, MAPF, CORIOLI, wdamp, dtl, dts,
                 ND_COEF, divdmp, fct, along, QA, ND_ORDER, QTRC, R, CV, CP, M):
    return _call("og_tstep_large", g, SCHEMES[scheme], SCHEMES[scheme_tracer],
                 st["DENS"], st["MOMZ"], st["MOMX"], st["MOMY"], st["RHOT"], QTRC, int(QA),
                 out["mflx_hi"], out["tflx_hi"], out["num_diff"],
                 tp["DENS_tp"], tp["MOMZ_tp"], tp["MOMX_tp"], tp["MOMY_tp"], tp["RHOT_tp"], tp.get("RHOQ_tp"),
                 CORIOLI, g.CDZ, g.CDX, g.CDY, g.FDZ, g.FDX, g.FDY, g.RCDZ, g.RCDX, g.RCDY, g.RFDZ, g.RFDX, g.RFDY,
                 ref["PHI"], GSQRT, J13G, J23G, 1.0, MAPF, R, CV, CP, M,
                 ref["REF_dens"], ref["REF_pott"], ref["REF_pres"], float(ND_COEF), int(ND_ORDER), 1.0, 1, wdamp,
                 float(divdmp),
                 int(fct), int(along), float(dtl), float(dts))


def max_residual(g, scheme, st, DPRES0, RT2P, num_diff, ref, REF_rhot, dtrk):
    return load().og_hevi_max_residual(
        C.byref(dims(g)), SCHEMES[scheme], _p(st["DENS"]), _p(st["MOMZ"]), _p(st["MOMX"]), _p(st["MOMY"]),
        _p(st["RHOT"]), _p(DPRES0), _p(RT2P), _p(num_diff), _p(g.CDZ), _p(g.FDZ), _p(g.FDX), _p(g.FDY), _p(g.RCDZ),
        _p(g.RCDX), _p(g.RCDY), _p(g.RFDZ), _p(g.RFDX), _p(g.RFDY), _p(ref["PHI"]), _p(ref["REF_dens"]),
        _p(REF_rhot), float(dtrk))


def domain_sum(g, var):
    return load().og_domain_sum(C.byref(dims(g)), _p(var), _p(g.CDZ), _p(g.CDX), _p(g.CDY))


def energy_sum(g, st, CZ):
    """Dry-air energy totals ENGT, ENGP, ENGK, ENGI [J] of a state dict."""
    out = np.zeros(4)
    load().og_energy_sum(C.byref(dims(g)), _p(st["DENS"]), _p(st["MOMZ"]), _p(st["MOMX"]), _p(st["MOMY"]),
                         _p(st["RHOT"]), _p(np.ascontiguousarray(CZ, dtype=np.float64)), _p(g.CDZ), _p(g.CDX),
                         _p(g.CDY), _p(out))
    return dict(zip(("ENGT", "ENGP", "ENGK", "ENGI"), (float(v) for v in out)))
