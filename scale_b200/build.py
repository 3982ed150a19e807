"""Build recipe of libscale_hevi.so (sm_100a) and of the CPU oracle library.

The CUDA library is compiled in-tree with nvcc directly (no JIT cache), so the
shared object travels with the repository snapshot to the GPU machine:

    python -m scale_b200.build            # build what is out of date
    python -m scale_b200.build --force    # rebuild everything

FP64 code is compiled with --fmad=false and the host code with
-ffp-contract=off: the kernels keep the reference's evaluation order without
fused multiply-adds so their results can be compared bit for bit with the
oracle, which the reference's GNU build flags also do not contract. The FP32
instantiations of the mixed-precision path (FLOAT_SOURCES, -DHEVI_FLOAT_TU)
compile with FMA contraction.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libscale_hevi.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "build" / "liboracle.so"

CU_SOURCES = ["capi.cu", "hevi_stage.cu", "hevi_tma.cu", "numfilter.cu", "tracer.cu", "misc.cu", "noalloc.cu",
              "persist.cu", "adjoint.cu"]
CPP_SOURCES = ["grid_coef.cpp"]
# The FP32 instantiations of the mixed-precision path compile a second time from
# these sources, with -DHEVI_FLOAT_TU and FMA contraction on: their results are
# held to a tolerance against the FP64 path, not bit for bit, so a*b+c may fuse.
FLOAT_SOURCES = ["hevi_stage.cu", "hevi_tma.cu", "numfilter.cu", "tracer.cu", "persist.cu"]
HEADERS = ["hevi_common.cuh", "hevi_stage.cuh", "hevi_kernels.cuh", "hevi_epilogue.cuh", "adjoint.cuh",
           "numfilter_body.cuh", "fill_body.cuh", "hevi_stage_body.cuh", "tma_util.cuh", "grid_coef.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> str:
    # the system compiler; an inherited CC/CXX wrapper may lack parts of the toolchain
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build_cuda(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in CU_SOURCES + CPP_SOURCES + HEADERS] + [ROOT / "include" / "scale_hevi.h", Path(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "--fmad=false", "--extended-lambda", "-lineinfo", "-ccbin", _host_cxx(),
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", str(ROOT / "include")]
    objs, cmds = [], []
    for src in CU_SOURCES + CPP_SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc, *common, *ARCH, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu") and verbose:
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd = [nvcc, *common, *ARCH, "-x", "c++", "-c", str(CSRC / src), "-o", str(obj)]
        cmds.append(cmd)
        objs.append(str(obj))
    f32 = [a for a in common if a != "--fmad=false"] + ["--fmad=true", "-DHEVI_FLOAT_TU"]
    for src in FLOAT_SOURCES:
        obj = objdir / (Path(src).stem + "_f32.o")
        cmds.append([nvcc, *f32, *ARCH, "-c", str(CSRC / src), "-o", str(obj)] + (["-Xptxas", "-v"] if verbose else []))
        objs.append(str(obj))
    # the translation units compile independently; the kernel templates make
    # some of them long, so they run side by side
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, c) for c in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs])
    tmp.replace(LIB)
    return LIB


def build_oracle(force: bool = False) -> Path:
    deps = list(ORACLE_DIR.glob("*.c")) + list(ORACLE_DIR.glob("*.h")) + [ORACLE_DIR / "Makefile"]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    _run(["make", "-C", str(ORACLE_DIR), "-B" if force else "all"])
    return ORACLE_LIB


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")
    if proc.stderr.strip():
        sys.stderr.write(proc.stderr)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    ap.add_argument("--no-oracle", action="store_true")
    a = ap.parse_args()
    print(build_cuda(a.force, a.verbose))
    if not a.no_oracle:
        print(build_oracle(a.force))


if __name__ == "__main__":
    main()
