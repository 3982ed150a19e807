"""Python binding of libscale_hevi.so.

The functions below carry the names and argument lists of the reference
procedures they replace (see include/scale_hevi.h). Arguments are passed by
keyword, as the reference's dummy names; arrays may be numpy arrays (host
entries) or torch CUDA tensors (device entries, ``*_dev`` functions), scalars
are Python numbers. Everything is handed to the C-ABI by reference, as
gfortran would. A nonzero status raises HeviError with the library's message,
mirroring the reference's PRC_abort.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np

from .build import LIB, ROOT

HEADER = ROOT / "include" / "scale_hevi.h"

ERRORS = {
    1: "SCALE_HEVI_ERR_ARG",
    2: "SCALE_HEVI_ERR_NOT_SETUP",
    3: "SCALE_HEVI_ERR_CUDA",
    4: "SCALE_HEVI_ERR_NONFINITE",
    5: "SCALE_HEVI_ERR_UNSUPPORTED",
    6: "SCALE_HEVI_ERR_ALLOC",
}


class HeviError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Index(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("KA", "IA", "JA", "KS", "KE", "IS", "IE", "JS", "JE", "KMAX", "IMAX", "JMAX",
                                       "KHALO", "IHALO", "JHALO", "IBLOCK", "JBLOCK")]


def header_functions() -> dict[str, list[str]]:
    """Exported functions declared in the header and their parameter names."""
    text = HEADER.read_text()
    macros = {}
    for m in re.finditer(r"#define\s+(SCALE_HEVI_\w+_ARGS)\s*\\\n((?:.*\\\n)*.*)\n", text):
        body = m.group(2).replace("\\\n", " ")
        macros[m.group(1)] = body
    out = {}
    for m in re.finditer(r"\n(?:int|void \*|const char \*|long long)\s*(\w+)\(([^;]*?)\);", text):
        name, params = m.group(1), m.group(2)
        for k, v in macros.items():
            params = params.replace(k, v)
        names = []
        for p in params.split(","):
            p = p.strip()
            if not p or p == "void":
                continue
            names.append(re.split(r"[\s\*]+", p)[-1])
        out[name] = names
    return out


_lib = None
_sig = None
# int (*)(void *const *fields, int nfields, int elem_bytes, void *user)
HALO_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_void_p)


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib, _sig
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run `python -m scale_b200.build` (or __graft_entry__.build())")
    lib = C.CDLL(str(p))
    _sig = header_functions()
    for name, params in _sig.items():
        f = getattr(lib, name)
        if name in ("scale_hevi_last_error", "scale_hevi_profile_report", "scale_hevi_autotune_report"):
            f.restype = C.c_char_p
        elif name == "scale_hevi_stream":
            f.restype = C.c_void_p
        elif name == "scale_hevi_kernel_launches":
            f.restype = C.c_longlong
        else:
            f.restype = C.c_int
        if name == "scale_hevi_setup":
            f.argtypes = [C.POINTER(Index), C.c_char_p, C.c_char_p, C.c_int]
        elif name == "scale_hevi_ensemble_setup":
            f.argtypes = [C.c_int, C.POINTER(Index), C.c_char_p, C.c_char_p, C.c_int]
        elif name == "scale_hevi_stage_shape":
            f.argtypes = [C.c_int, C.c_int]
        elif name in ("scale_hevi_short_type", "scale_hevi_tinteg_short_type"):
            f.argtypes = [C.c_char_p]
        elif name == "scale_hevi_set_halo_exchange":
            f.argtypes = [HALO_FN, C.c_void_p]
        elif name in ("scale_hevi_stage_autotune", "scale_hevi_numfilter_form", "scale_hevi_tracer_fct_form"):
            f.argtypes = [C.c_int]
        elif name == "scale_hevi_stage_shape_get":
            f.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
        elif name == "scale_hevi_profile":
            f.argtypes = [C.c_int]
        elif name in ("scale_hevi_capture_begin", "scale_hevi_capture_end"):
            f.argtypes = []
        else:
            f.argtypes = [C.c_void_p] * len(params)
    _lib = lib
    return lib


def last_error() -> str:
    return load().scale_hevi_last_error().decode()


def _check(rc: int) -> None:
    if rc != 0:
        raise HeviError(rc, last_error())


class _Args:
    """Marshals keyword arguments into by-reference C arguments, keeping the
    temporaries alive for the duration of the call."""

    def __init__(self):
        self.keep = []

    def ptr(self, v, ints: bool):
        if v is None:
            return None
        if isinstance(v, np.ndarray):
            if v.dtype == np.float64 and (v.flags.f_contiguous or v.flags.c_contiguous):
                return v.ctypes.data
            raise TypeError("arrays must be contiguous float64 in Fortran order")
        if hasattr(v, "data_ptr"):  # torch tensor
            return v.data_ptr()
        if isinstance(v, (bool, np.bool_)) or (ints and isinstance(v, (int, np.integer))):
            c = C.c_int(int(v))
        else:
            c = C.c_double(float(v))
        self.keep.append(c)
        return C.addressof(c)


INT_ARGS = {"FLAG_FCT_MOMENTUM", "FLAG_FCT_T", "FLAG_FCT_ALONG_STREAM", "FLAG_FCT_TRACER", "BND_W", "BND_E",
            "BND_S", "BND_N", "last", "ND_ORDER", "ND_USE_RS", "QA", "nfields", "n", "extra_arrivals"}
# arguments passed as they are (an address, a C string or a stream handle), not by reference
RAW_ARGS = {"idx", "flux_type", "stream"}


def call(name: str, **kw) -> None:
    """Call an exported entry by name with keyword arguments named as its dummies."""
    lib = load()
    params = _sig[name]
    unknown = set(kw) - set(params)
    if unknown:
        raise TypeError(f"{name}: unknown arguments {sorted(unknown)}")
    a = _Args()
    args = [kw.get(p) if p in RAW_ARGS else a.ptr(kw.get(p), p in INT_ARGS) for p in params]
    _check(getattr(lib, name)(*args))


# ---- library state ----------------------------------------------------------------
def setup(index: dict, flux_type: str = "UD3", flux_tracer_type: str = "UD3", device: int = 0) -> None:
    """ATMOS_DYN_FVM_flux_setup + index setup of the HEVI short step."""
    lib = load()
    idx = Index(**index)
    _check(lib.scale_hevi_setup(C.byref(idx), flux_type.encode(), flux_tracer_type.encode(), int(device)))


def ensemble_setup(indices: list[dict], flux_type: str = "UD3", flux_tracer_type: str = "UD3",
                   device: int = 0) -> dict[str, np.ndarray]:
    """Set up an ensemble of len(indices) members; returns its pooled layout
    (ensemble_layout())."""
    lib = load()
    arr = (Index * len(indices))(*[Index(**d) for d in indices])
    _check(lib.scale_hevi_ensemble_setup(len(indices), arr, flux_type.encode(), flux_tracer_type.encode(),
                                         int(device)))
    return ensemble_layout(len(indices))


def ensemble_layout(n: int) -> dict[str, np.ndarray]:
    """Offsets of each member in the pooled arrays: cell0 (3-D fields), col0
    (2-D fields), z0/x0/y0 (1-D vectors); n+1 entries, the last the totals."""
    out = {k: np.zeros(n + 1, dtype=np.int64) for k in ("cell0", "col0", "z0", "x0", "y0")}
    ptr = lambda v: v.ctypes.data_as(C.POINTER(C.c_longlong))  # noqa: E731
    _check(load().scale_hevi_ensemble_layout(*(ptr(out[k]) for k in ("cell0", "col0", "z0", "x0", "y0"))))
    return out


def pool(arrays: list[np.ndarray], offsets: np.ndarray, ncomp: int = 1, slots: list[int] | None = None) -> np.ndarray:
    """Pooled array of per-member arrays (Fortran order): component q of member
    m at q*offsets[-1] + offsets[m]. For 1-D vectors, `slots` gives each
    member's length in the pool (a shorter vector leaves its last slot zero)."""
    total = int(offsets[-1])
    out = np.zeros(ncomp * total)
    for m, a in enumerate(arrays):
        flat = np.ravel(a, order="F")
        n = flat.size // ncomp
        if slots is not None and n > slots[m]:
            raise ValueError(f"member {m}: {n} values for {slots[m]} slots")
        for q in range(ncomp):
            o = q * total + int(offsets[m])
            out[o:o + n] = flat[q * n:(q + 1) * n]
    return out


def unpool(pooled: np.ndarray, offsets: np.ndarray, shapes: list[tuple], ncomp: int = 1) -> list[np.ndarray]:
    """Per-member arrays (Fortran order, shape shapes[m] + (ncomp,) when
    ncomp > 1) of a pooled array."""
    total = int(offsets[-1])
    flat = np.asarray(pooled).ravel()
    out = []
    for m, shp in enumerate(shapes):
        n = int(np.prod(shp))
        comps = [flat[q * total + int(offsets[m]): q * total + int(offsets[m]) + n] for q in range(ncomp)]
        v = np.concatenate(comps) if ncomp > 1 else comps[0].copy()
        out.append(v.reshape(tuple(shp) + ((ncomp,) if ncomp > 1 else ()), order="F"))
    return out


def short_type(name: str = "HEVI") -> None:
    """The short step the RK4 entries and the large step run: "HEVI" or "HEVE"
    (ATMOS_DYN_Tstep_short_regist)."""
    _check(load().scale_hevi_short_type(name.encode()))


def tinteg_short_type(name: str = "RK4") -> None:
    """The short integrator the large step and the RK3 entries run: "RK4",
    "RK3" (Heun) or "RK3WS2002" (ATMOS_DYN_Tinteg_short_setup)."""
    _check(load().scale_hevi_tinteg_short_type(name.encode()))


_halo_cb = None  # the registered callback object, kept alive while set


def set_halo_exchange(fn) -> None:
    """Register fn(ptrs, nfields, elem_bytes) -> None as the lateral halo
    exchange of every halo fill (None restores the periodic fill); ptrs are
    the device addresses of the (KA,IA,JA) fields (scale_hevi_set_halo_exchange)."""
    global _halo_cb
    if fn is None:
        _check(load().scale_hevi_set_halo_exchange(HALO_FN(), None))
        _halo_cb = None  # finalize() clears the library's hook as well
        return

    def tramp(fields, nfields, elem_bytes, user):
        try:
            fn([fields[q] for q in range(nfields)], nfields, elem_bytes)
            return 0
        except Exception:  # reported to the library as a failed exchange
            import traceback

            traceback.print_exc()
            return 1

    cb = HALO_FN(tramp)
    _check(load().scale_hevi_set_halo_exchange(cb, None))
    _halo_cb = cb


def stage_shape(tile_x: int = 0, raster: int = 0) -> None:
    """Tile width and raster height of the stage kernel (0: defaults)."""
    _check(load().scale_hevi_stage_shape(int(tile_x), int(raster)))


def stage_autotune(enable: bool = True) -> None:
    """Tune the stage shape at the next short-step call of each path."""
    _check(load().scale_hevi_stage_autotune(int(bool(enable))))


def stage_shape_get(mixed: bool = False) -> tuple[int, int]:
    tx, r = C.c_int(), C.c_int()
    _check(load().scale_hevi_stage_shape_get(C.byref(tx), C.byref(r), int(bool(mixed))))
    return tx.value, r.value


def autotune_report() -> dict:
    import json

    t = load().scale_hevi_autotune_report().decode()
    return json.loads(t) if t else {}


def finalize() -> None:
    load().scale_hevi_finalize()


def check() -> None:
    _check(load().scale_hevi_check())


def kernel_launches() -> int:
    return int(load().scale_hevi_kernel_launches())


def transfer_bytes() -> tuple[int, int]:
    """(host->device, device->host) bytes staged by the host-array entries since setup."""
    h, d = C.c_longlong(0), C.c_longlong(0)
    _check(load().scale_hevi_transfer_bytes(C.byref(h), C.byref(d)))
    return int(h.value), int(d.value)


def capture_begin() -> None:
    """Start recording the _dev calls on the library stream into a CUDA graph."""
    _check(load().scale_hevi_capture_begin())


def capture_end() -> None:
    _check(load().scale_hevi_capture_end())


def replay(n: int = 1) -> None:
    """Launch the captured graph n times on the library stream."""
    call("scale_hevi_replay", n=n)


def profile(enable: bool) -> None:
    """Enable (and reset) or disable the per-section CUDA-event timers."""
    _check(load().scale_hevi_profile(1 if enable else 0))


def profile_report() -> dict:
    """{section: (launches, total_ms)} since the last profile(True)."""
    import json

    return {k: (int(v[0]), float(v[1])) for k, v in json.loads(load().scale_hevi_profile_report().decode()).items()}


def boundary_dev(DENS, MOMZ, MOMX, MOMY, RHOT) -> None:
    """Vertical boundary values and periodic halo of the five prognostic fields."""
    call("scale_hevi_boundary_dev", DENS=DENS, MOMZ=MOMZ, MOMX=MOMX, MOMY=MOMY, RHOT=RHOT)


def stream_handle() -> int:
    return int(load().scale_hevi_stream() or 0)


# ---- reference-named entries (host arrays) ---------------------------------------
def ATMOS_DYN_Tstep_short_fvm_hevi(**kw):
    call("ATMOS_DYN_Tstep_short_fvm_hevi_b200", **kw)


def ATMOS_DYN_Tstep_short_fvm_heve(**kw):
    call("ATMOS_DYN_Tstep_short_fvm_heve_b200", **kw)


def ATMOS_DYN_Tinteg_short_rk4(**kw):
    call("ATMOS_DYN_Tinteg_short_rk4_b200", **kw)


def ATMOS_DYN_Tinteg_short_rk3(**kw):
    call("ATMOS_DYN_Tinteg_short_rk3_b200", **kw)


def ATMOS_DYN_numfilter_coef(**kw):
    call("ATMOS_DYN_numfilter_coef_b200", **kw)


def ATMOS_DYN_Tstep_tracer_fvm_heve(**kw):
    call("ATMOS_DYN_Tstep_tracer_fvm_heve_b200", **kw)


def ATMOS_DYN_Tinteg_tracer_rk3(**kw):
    call("ATMOS_DYN_Tinteg_tracer_rk3_b200", **kw)


def ATMOS_DYN_Tstep_large_fvm_heve(**kw):
    call("ATMOS_DYN_Tstep_large_fvm_heve_b200", **kw)


def ATMOS_DYN_divergence(**kw):
    call("ATMOS_DYN_divergence_b200", **kw)


# ---- device-array entries -----------------------------------------------------------
def ATMOS_DYN_Tstep_short_fvm_hevi_dev(**kw):
    call("ATMOS_DYN_Tstep_short_fvm_hevi_b200_dev", **kw)


def ATMOS_DYN_Tstep_short_fvm_heve_dev(**kw):
    call("ATMOS_DYN_Tstep_short_fvm_heve_b200_dev", **kw)


def ATMOS_DYN_Tinteg_short_rk4_dev(**kw):
    call("ATMOS_DYN_Tinteg_short_rk4_b200_dev", **kw)


def ATMOS_DYN_Tinteg_short_rk3_dev(**kw):
    call("ATMOS_DYN_Tinteg_short_rk3_b200_dev", **kw)


def ATMOS_DYN_numfilter_coef_dev(**kw):
    call("ATMOS_DYN_numfilter_coef_b200_dev", **kw)


def short_step_persistent_dev(**kw):
    """Numerical filter + RK4 HEVI + boundary values and halo of every member
    as one persistent launch (scale_hevi_short_step_persistent_dev)."""
    call("scale_hevi_short_step_persistent_dev", **kw)


def short_step_persistent_mixed_dev(**kw):
    call("scale_hevi_short_step_persistent_mixed_dev", **kw)


def persistent_wait(seconds: float, extra_arrivals: int = 0) -> None:
    """Time limit of the persistent step's grid barriers; extra_arrivals = 1
    makes them wait for a CTA that does not exist (a test of the limit)."""
    call("scale_hevi_persistent_wait", seconds=seconds, extra_arrivals=extra_arrivals)


def numfilter_form(tiled: bool) -> None:
    """The filter's tiled form (True, the default) or the column kernel for one domain."""
    _check(load().scale_hevi_numfilter_form(int(bool(tiled))))


def tracer_fct_form(fused: bool) -> None:
    """The FCT-limited tracer stage's fused form (True, the default) or the
    three-kernel form."""
    _check(load().scale_hevi_tracer_fct_form(int(bool(fused))))


def persistent_grid() -> int:
    """CTAs of the last persistent launch."""
    n = C.c_int(0)
    _check(load().scale_hevi_persistent_grid(C.byref(n)))
    return n.value


def ATMOS_DYN_Tstep_tracer_fvm_heve_dev(**kw):
    call("ATMOS_DYN_Tstep_tracer_fvm_heve_b200_dev", **kw)


def ATMOS_DYN_Tinteg_tracer_rk3_dev(**kw):
    call("ATMOS_DYN_Tinteg_tracer_rk3_b200_dev", **kw)


def ATMOS_DYN_Tinteg_tracer_rk3_mixed_dev(**kw):
    """Tracer RK3 with FP32 flux and limiter arithmetic: float32 mflx_hi,
    num_diff and RHOQ_t; float64 tracer and densities (device arrays)."""
    call("ATMOS_DYN_Tinteg_tracer_rk3_b200_mixed_dev", **kw)


def ATMOS_DYN_Tstep_large_fvm_heve_dev(**kw):
    call("ATMOS_DYN_Tstep_large_fvm_heve_b200_dev", **kw)


def ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(index: dict, flux_type: str, stream: int, **kw):
    """One HEVI stage that allocates no device memory (no scale_hevi_setup needed);
    device arrays as in ATMOS_DYN_Tstep_short_fvm_hevi_dev, stream a cudaStream_t handle."""
    idx = Index(**index)
    call("ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc", idx=C.addressof(idx), flux_type=flux_type.encode(),
         stream=int(stream), **kw)


def ATMOS_DYN_divergence_dev(**kw):
    call("ATMOS_DYN_divergence_b200_dev", **kw)


def ATMOS_DYN_Tinteg_short_rk4_mixed_dev(**kw):
    """Mixed-precision RK4 short step; mflx_hi, tflx_hi, *_t, num_diff, DDIV are float32 device tensors."""
    call("ATMOS_DYN_Tinteg_short_rk4_b200_mixed_dev", **kw)


def ATMOS_DYN_numfilter_coef_mixed_dev(**kw):
    """Numerical filter with a float32 num_diff device tensor."""
    call("ATMOS_DYN_numfilter_coef_b200_mixed_dev", **kw)


def COMM_vars8_dev(var, nfields: int):
    call("COMM_vars8_b200_dev", var=var, nfields=nfields)


def domain_sum_dev(var, CDZ, CDX, CDY) -> float:
    out = np.zeros(1)
    call("scale_hevi_domain_sum_dev", var=var, CDZ=CDZ, CDX=CDX, CDY=CDY, total=out)
    return float(out[0])


def energy_sum_dev(DENS, MOMZ, MOMX, MOMY, RHOT, CZ, CDZ, CDX, CDY) -> dict:
    """FP64 domain totals of the dry-air energies [J]: ENGT, ENGP, ENGK, ENGI."""
    out = np.zeros(4)
    call("scale_hevi_energy_sum_dev", DENS=DENS, MOMZ=MOMZ, MOMX=MOMX, MOMY=MOMY, RHOT=RHOT, CZ=CZ, CDZ=CDZ,
         CDX=CDX, CDY=CDY, totals=out)
    return dict(zip(("ENGT", "ENGP", "ENGK", "ENGI"), (float(v) for v in out)))
