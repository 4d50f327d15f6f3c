"""Build step of the package: compiles csrc/*.cu for sm_100a into
liberebus_b200.so next to this file (in-tree, so the library travels with
the source tree)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liberebus_b200.so")
SOURCES = ["api.cu", "markers.cu", "stencils.cu", "assemble.cu", "bandlu.cu", "mfront.cu",
           "adjoint.cu", "krylov.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # every a*b+c rounds twice, as in the reference; the LU calls fma()
    "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
    "-Xptxas", "-v",
]


def build(force=False, verbose=False):
    srcs = [os.path.join(SRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(SRC, h) for h in os.listdir(SRC) if h.endswith((".cuh", ".h"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "erebus_b200.h"))
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps)):
        return LIB
    cmd = [NVCC] + FLAGS + srcs + ["-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stderr[-6000:])
        raise RuntimeError("nvcc failed (see %s)" % log)
    if verbose:
        sys.stdout.write(r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
