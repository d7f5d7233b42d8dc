"""Build libselfgpu.so (the CUDA engine and its C ABI) in-tree for sm_100a.

Run ``python -m self_b200.build`` (or ``__graft_entry__.build()``).  The
library lands next to this file so that it travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libselfgpu.so")
BUILD_DIR = os.path.join(HERE, "_build")

# (source, extra flags): the reference-rounding FP64 kernels (drop-in wrappers,
# the SELFGPU_FP64_REF stage form, the FP64 closure) are built without
# multiply-add contraction so their roundings follow the reference's CPU path
# exactly; the production FP64 stage form (stage_fp64_prod.cu) contracts.
SOURCES = [("setup_host.cpp", []), ("legacy_ops.cu", ["-fmad=false"]), ("stage_fp64.cu", ["-fmad=false"]),
           ("stage_fp64_prod.cu", []), ("stage_fp32.cu", []), ("engine.cu", []), ("noalloc.cu", ["-fmad=false"]),
           ("mlp.cu", []), ("checkpoint.cpp", []), ("decomp.cpp", []), ("hip_shim.cpp", [])]
HEADERS = ["selfgpu_internal.h", "physics.cuh", "fused_stage.cuh", "fused_stage_tma.cuh", "stage_dispatch.cuh",
           "av_closure.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(BUILD_DIR, exist_ok=True)
    inc = os.path.join(HERE, "..", "include")
    deps_common = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(inc, "selfgpu.h")]
    objs = []
    jobs = []
    for src, extra in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + deps_common):
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-I", inc, "-c", s, "-o", o]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            jobs.append((cmd, src))
    procs = []
    for cmd, src in jobs:
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or (verbose and out):
            sys.stdout.write(out.decode(errors="replace"))
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(OUT, objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
