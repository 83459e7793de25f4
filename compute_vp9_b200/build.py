"""Build the native libraries in-tree (sm_100a; nvcc cross-compiles without a GPU).

    python -m compute_vp9_b200.build            # product + synth
    python -m compute_vp9_b200.build --oracle   # also the CPU checkers (oracle/)

Outputs under compute_vp9_b200/lib/:
    libcvp9_cuda.so   kernels + C host backend (the product, C ABI)
    libcvp9_synth.so  seeded synthetic parsed-frame generator (host C)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
INC = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_C = ["backend_common.c", "cuda_backend.c", "batch.c", "pack.c", "hbd.c"]
CUDA_SRC = ["recon.cu", "recon_static.cu"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, oracle=False, verbose_ptxas=False):
    os.makedirs(LIB, exist_ok=True)
    objdir = os.path.join(LIB, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    incs = ["-I" + INC, "-I" + CSRC, "-I" + os.path.join(CUDA_HOME, "include")]

    objs = []
    for src in CUDA_SRC:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        if force or _newer(o, [s] + headers):
            cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            _run(cmd + incs + ["-c", s, "-o", o])
        objs.append(o)
    for src in HOST_C:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(objdir, src + ".o")
        if force or _newer(o, [s] + headers):
            _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-ffp-contract=off", "-Wall",
                  "-Wno-unused-function"] + incs + ["-c", s, "-o", o])
        objs.append(o)
    so = os.path.join(LIB, "libcvp9_cuda.so")
    if force or _newer(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", so] + objs +
             ["-lpthread", "-lm", "-ldl", "-lrt"])

    synth_src = os.path.join(CSRC, "synth.c")
    synth_so = os.path.join(LIB, "libcvp9_synth.so")
    if force or _newer(synth_so, [synth_src] + headers):
        _run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", "-Wall", "-I" + INC,
              "-o", synth_so, synth_src])

    if oracle:
        build_oracle()
    return so


def build_oracle():
    """Compile oracle/ (restatements) and, where the reference tree is present,
    oracle/_ref (the reference's own CPU reconstruction built from source) and
    the drop-in harness (the reference library with the CUDA branch,
    integration/)."""
    _run(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    _run(["make", "-s", "-C", os.path.join(ROOT, "integration")])


if __name__ == "__main__":
    build(force="--force" in sys.argv, oracle="--oracle" in sys.argv,
          verbose_ptxas="--ptxas" in sys.argv)
