"""Build libbx200.so in-tree with nvcc for sm_100a.

The FP64 stage kernels and the per-block kernels are compiled with
--fmad=false: the reference's arithmetic is not contracted into fused
multiply-adds, so the GPU FP64 path keeps the reference operation order.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libbx200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr"]
# (source, extra flags)
UNITS = [
    ("bx_stage_fp64.cu", ["--fmad=false"]),
    ("bx_compat.cu", ["--fmad=false"]),
    ("bx_stage_fp32.cu", []),
    ("bx_stage3d.cu", []),
    ("bx_stage3d_fpt2.cu", []),
    ("bx_stage3d_v2.cu", []),
    ("bx_amr.cu", []),
    ("bx_amr_plan.cu", []),
    ("bx_implicit.cu", ["--fmad=false"]),
    ("bx_learned.cu", []),
    ("bx_noalloc.cu", []),
    ("bx_heat.cu", []),
    ("bx_tune.cu", []),
    ("bx_capi.cu", []),
]
HEADERS = ["bx_physics.cuh", "bx_stage.cuh", "bx_device.h", "bx_stage3d.cuh", "bx_stage3d_v2.cuh", "bx_stage3d_launch.cuh", "bx_tma.cuh", "bx_core.h",
           "bx_impl_kernels.cuh", "bx_krylov.cuh", "bx_tune.h", "bx_tc.cuh", "bx_learned.cuh", "bx_learned_kernels.cuh", "bx_amr.h"]


def _sources_newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, force=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "bx200.h")]
    objs = []
    jobs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _sources_newer(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + COMMON + flags + ["-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _sources_newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
