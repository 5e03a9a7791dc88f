"""Builds libtidegbm_b200.so in-tree for sm_100a (nvcc + g++, no JIT cache).

    python -m tidegbm_b200.build        # or tidegbm_b200.build.build()

Objects go to tidegbm_b200/_build/; the shared library to tidegbm_b200/.
Files whose FP64 arithmetic must follow the reference's statement order
(split gains, pairwise gradients, quantile edges) are compiled with -fmad=false; host code with
-ffp-contract=off.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtidegbm_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NO_FMA = {"kernels_split.cu", "kernels_obj.cu", "kernels_post.cu", "kernels_binfit.cu", "kernels_wave_scan.cu"}


def _cuda_home() -> str:
    env = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if env:
        return env
    nvcc = shutil.which("nvcc")
    return os.path.dirname(os.path.dirname(nvcc)) if nvcc else "/usr/local/cuda"


def _sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, nvcc: str, cuda_inc: str) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))] + [
        os.path.join(INCLUDE, "tidegbm_b200.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    if src.endswith(".cu"):
        cmd = [nvcc, "-O3", "-std=c++17", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I", CSRC,
               "-I", INCLUDE,
               "-c", path, "-o", obj]
        if src in NO_FMA:
            cmd.insert(1, "-fmad=false")
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fvisibility=hidden", "-pthread",
               "-I", CSRC, "-I", INCLUDE, "-I", cuda_inc, "-c", path, "-o", obj]
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    home = _cuda_home()
    nvcc = os.path.join(home, "bin", "nvcc")
    if not os.path.exists(nvcc):
        nvcc = shutil.which("nvcc") or nvcc
    cuda_inc = os.path.join(home, "include")
    srcs = _sources()
    with ThreadPoolExecutor(max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, nvcc, cuda_inc), srcs))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    tmp = LIB + ".tmp"
    subprocess.run([nvcc, "-shared", *ARCH, "-cudart", "static", "-o", tmp, *objs, "-lpthread"], check=True)
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
