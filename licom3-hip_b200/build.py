"""Build recipe for liblicom_tracer.so (sm_100a) and the CPU checker libraries.

Usage: python licom3-hip_b200/build.py [--oracle [--ref <reference source tree>]]

The CUDA library is compiled per translation unit with nvcc for
``arch=compute_100a,code=sm_100a``; files whose results are compared bit for
bit with the FP64 oracle are compiled with ``-fmad=false``.
"""
import os
import subprocess
import sys
import shutil

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblicom_tracer.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "--expt-relaxed-constexpr", "-I" + os.path.join(REPO, "include")]
# translation unit -> extra flags
CU_UNITS = {
    "lt_api.cu": [],
    "lt_step_fp64.cu": ["-fmad=false"],
    "lt_step_mixed.cu": [],
    "lt_misc.cu": ["-fmad=false"],
    "lt_noalloc.cu": ["-fmad=false"],
    "lt_batch.cu": [],
    "lt_serve.cu": [],
    "lt_turb.cu": ["-fmad=false"],
    "lt_del4u.cu": ["-fmad=false"],
    "lt_restart.cu": [],
}
CPP_UNITS = ["lt_synth_api.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError("build step failed: " + os.path.basename(cmd[-1]))
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + [
        os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))]


def build_cuda(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    hdrs = _headers()
    for unit, extra in CU_UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, unit + ".o")
        if _stale(obj, [src] + hdrs) or ptxas_info:
            cmd = [NVCC] + ARCH + NVFLAGS + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", "-o", obj, src]
            out = _run(cmd)
            if verbose or ptxas_info:
                sys.stdout.write(out)
        objs.append(obj)
    for unit in CPP_UNITS:
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit + ".o")
        if _stale(obj, [src] + hdrs):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-c", "-o", obj, src])
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "--cudart", "static", "-o", LIB] + objs)
    return LIB


def build_oracle(ref=None):
    """CPU checker libraries (test infrastructure): the oracle and the host
    input generator; with ``ref`` (or LICOM_REFERENCE_DIR), the directory of
    the reference's sources, also the reference's own tracer.cpp, convadj.cpp,
    icesnow.cpp and readyc.cpp compiled for the CPU."""
    oracle_dir = os.path.join(REPO, "oracle")
    env = dict(os.environ)
    env.pop("CXX", None)
    targets = ["all"]
    ref_tree = ref or os.environ.get("LICOM_REFERENCE_DIR")
    args = []
    if ref_tree and os.path.isfile(os.path.join(ref_tree, "tracer.cpp")):
        targets.append("ref")
        args.append("REF=" + ref_tree)
    subprocess.run(["make", "-s", "-C", oracle_dir] + args + targets, check=True, env=env)


if __name__ == "__main__":
    build_cuda(verbose=True, ptxas_info="--ptxas" in sys.argv)
    if "--oracle" in sys.argv:
        build_oracle(sys.argv[sys.argv.index("--ref") + 1] if "--ref" in sys.argv else None)
    print(LIB)
