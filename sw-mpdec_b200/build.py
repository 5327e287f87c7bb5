"""Build libswm.so (the sm_100a C-ABI library) in place with nvcc.

Translation units and their floating-point flags:
  swm_kernels.cu    -fmad=false  (Patankar assembly, Jacobi, dt, layouts)
  swm_rhs_exact.cu  -fmad=false  (RHS, reference expression order; FP64 ensemble step)
  swm_rhs_fast.cu   default      (RHS, FP64 with contraction and the split form;
                                  their ensemble steps)
  swm_capi.cu       host orchestration, C ABI
  swm_batch.cu      batched ensembles
  swm_noalloc.cu    allocation-free Jacobi entry point
  swm_ic.cu         -fmad=false  (initial conditions, L1 error)
  swm_output.cu     -fmad=false  (formatted solution files)
Usage: python sw-mpdec_b200/build.py [--verbose] [--force] [--ptxas] [--checked]
(--checked: libswm_checked.so with device-side index checks, for tests)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libswm.so")
# the checked build: device-side index checks at the wrapped-index sites (SWM_IN_RANGE),
# failures recorded instead of faulting; for tests, never loaded by the product path
BUILD_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libswm_checked.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I" + os.path.join(HERE, "..", "include")]
UNITS = [
    ("swm_kernels.cu", ["-fmad=false"]),
    ("swm_rhs_exact.cu", ["-fmad=false"]),
    ("swm_rhs_fast.cu", []),
    ("swm_capi.cu", ["-Xcompiler", "-ffp-contract=off"]),
    ("swm_batch.cu", []),
    ("swm_noalloc.cu", []),
    ("swm_ic.cu", ["-fmad=false"]),
    ("swm_output.cu", ["-fmad=false"]),
]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(HERE, "..", "include", "swm.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False, ptxas_verbose=False, checked=False):
    bdir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    extra = ["-DSWM_CHECKED"] if checked else []
    os.makedirs(bdir, exist_ok=True)
    objs = []
    hdrs = _headers()
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(bdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, *COMMON, *extra, *flags, "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(lib, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", lib, *objs, "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv,
                ptxas_verbose="--ptxas" in sys.argv, checked="--checked" in sys.argv))
