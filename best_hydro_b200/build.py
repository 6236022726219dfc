"""Builds libbestgpu (the sm_100a CUDA kernels and the C ABI) in-tree, into best_hydro_b200/lib/.

Run as ``python -m best_hydro_b200.build`` or through ``__graft_entry__.build()``.  nvcc cross-compiles
for sm_100a without a GPU.  The assembly is compiled with -fmad=false (BEST's -ffp-contract=off);
everything else may contract.  Objects are rebuilt when a source or header is newer.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(LIBDIR, "obj")
LIB = os.path.join(LIBDIR, "libbestgpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", f"-I{CSRC}", f"-I{os.path.join(ROOT, 'include')}"]
# (source, extra flags)
SOURCES = [
    ("assemble.cu", ["-fmad=false"]),
    ("assemble_fast.cu", []),
    ("geometry.cu", ["-fmad=false"]),
    ("lu.cu", []),
    ("solve.cu", []),
    ("tc_gemm.cu", []),
    ("mixed.cu", []),
    ("hmatrix.cu", ["-fmad=false"]),
    ("adjoint.cu", []),
    ("api.cpp", []),
    ("driver.cpp", []),
]
# host programs linked against the library: (source, output name)
PROGRAMS = [("best_gpu_main.cpp", "best_gpu")]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(verbose=False):
    os.makedirs(OBJDIR, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src.rsplit(".", 1)[0] + ".o")
        objs.append(o)
        if _newer(o, [s, __file__] + hdrs):
            lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
            _run([NVCC] + ARCH + COMMON + extra + lang + ["-c", s, "-o", o], verbose)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs, verbose)
    for src, name in PROGRAMS:
        s = os.path.join(CSRC, src)
        exe = os.path.join(LIBDIR, name)
        if _newer(exe, [s, LIB] + hdrs):
            _run(["g++", "-O2", "-std=c++17", f"-I{os.path.join(ROOT, 'include')}", "-o", exe, s, f"-L{LIBDIR}",
                  "-lbestgpu", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
