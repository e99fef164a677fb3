"""Build the CUDA C-ABI library ``flash5_b200/_flash_hy.so`` for sm_100a.

``hy_variant.cu`` is compiled once per arithmetic variant: FP64 without FMA
contraction (the parity path), FP64 with FMA, and FP32 reconstruction with
FP64 update (three units, one per threads-per-CTA candidate of its direction
kernels).  Objects go to ``flash5_b200/_build``; the shared library is
written in-tree so that it travels with the repository snapshot.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "_flash_hy.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                 "-ccbin", "g++"]

# The FP32 arithmetic of the mixed units (reconstruction, species face
# values, the learned guess): approximate FP32 division and square root,
# FP32 denormals flushed.  FP64 arithmetic is unaffected by these flags.
FP32_FAST = ["-ftz=true", "-prec-div=false", "-prec-sqrt=false"]

UNITS = [
    ("hy_fp64_exact.o", "hy_variant.cu", ["-DFHY_VARIANT=1", "--fmad=false"]),
    ("hy_fp64_fma.o", "hy_variant.cu", ["-DFHY_VARIANT=2", "--fmad=true"]),
    ("hy_mixed0.o", "hy_variant.cu", ["-DFHY_VARIANT=3", "-DFHY_MXSEL=0", "--fmad=true"] + FP32_FAST),
    ("hy_mixed1.o", "hy_variant.cu", ["-DFHY_VARIANT=3", "-DFHY_MXSEL=1", "--fmad=true"] + FP32_FAST),
    ("hy_mixed2.o", "hy_variant.cu", ["-DFHY_VARIANT=3", "-DFHY_MXSEL=2", "--fmad=true"] + FP32_FAST),
    ("flash_hy.o", "flash_hy.cu", ["--fmad=false"]),
    ("riemann_exact.o", "riemann_exact.cu", ["--fmad=true"] + FP32_FAST),
    ("cfl_noalloc.o", "cfl_noalloc.cu", ["--fmad=false"]),
    ("spec.o", "spec.cu", ["--fmad=false"]),
    ("spec_mx.o", "spec.cu", ["-DFHY_SPEC_MIXED", "--fmad=true"] + FP32_FAST),
    ("refine.o", "refine.cu", ["--fmad=false"]),
    ("tree.o", "tree.cu", []),
    ("tree_dev.o", "tree_dev.cu", []),
]


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "flash_hy.h"))
    objs = []
    procs = []
    for obj, src, flags in UNITS:
        o = os.path.join(BUILD, obj)
        s = os.path.join(CSRC, src)
        objs.append(o)
        cmd = [NVCC] + COMMON + flags + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", s, "-o", o]
        stamp = o + ".cmd"
        same = os.path.exists(stamp) and open(stamp).read() == " ".join(cmd)
        if force or not same or _stale(o, [s] + headers):
            with open(stamp, "w") as f:
                f.write(" ".join(cmd))
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out)
        if (verbose or ptxas_info) and out:
            print(out, file=sys.stderr)
    if force or _stale(OUT, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, force="-f" in sys.argv)
