"""Builds colvillea_b200/libcolvillea_b200.so for sm_100a with nvcc.

The library is compiled with IEEE FP32 arithmetic and no multiply-add
contraction (-fmad=false, default -prec-div/-prec-sqrt): the per-sample
arithmetic follows the reference's source order, so that results can be
compared with the CPU oracle at the ulp level.  Traversal arithmetic that
wants fused multiply-adds uses explicit __fmaf_rn.

    python -m colvillea_b200.build          # or build() from Python
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcolvillea_b200.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["cl_units.cu", "cl_texture.cu", "cl_bvh_build.cu", "cl_dome.cu", "cl_guide.cu", "cl_integrator.cu", "cl_capi.cu", "cl_io.cpp"]
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _compile(src):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(HERE, "..", "include", "colvillea_b200.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps) \
            and os.path.getmtime(obj) >= os.path.getmtime(__file__):
        return obj, ""
    cmd = [NVCC, *ARCH, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(_compile, SOURCES))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log.strip():
                print(log, file=sys.stderr)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
