"""Build the B200 flexible-dual-grid library and its torch extension in-tree.

* ``lib/libovx_fdg.so``   -- CUDA kernels + C ABI (include/ovx_fdg.h), sm_100a only.
* ``o_voxel/_C<EXT_SUFFIX>`` -- torch extension (csrc/ext.cpp) linked against it.

``-fmad=false`` is part of the contract: the kernels reproduce the reference
CPU arithmetic operation by operation, which an FMA contraction would change.
"""
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
INCLUDE = os.path.join(REPO, "include")
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libovx_fdg.so")
EXT = os.path.join(PKG, "o_voxel", "_C" + sysconfig.get_config_var("EXT_SUFFIX"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(*names):
    return [os.path.join(CSRC, n) for n in names] + [os.path.join(INCLUDE, "ovx_fdg.h")]


def build_lib(force=False, verbose=False):
    srcs = _sources("fdg_kernels.cu", "fdg_mesh.cu", "fdg_device.cuh")
    if not (force or _newer(LIB, srcs)):
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [NVCC, *ARCH, *NVCC_FLAGS, "-shared", "-I", INCLUDE, srcs[0], srcs[1], "-o", LIB]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    subprocess.check_call(cmd)
    return LIB


def build_ext(force=False):
    srcs = _sources("ext.cpp") + [LIB]
    if not (force or _newer(EXT, srcs)):
        return EXT
    import torch
    from torch.utils import cpp_extension as ce

    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w",
           f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-DTORCH_EXTENSION_NAME=_C", "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-I", INCLUDE, "-I", os.path.join(cuda_home, "include"), "-I", sysconfig.get_paths()["include"]]
    for p in ce.include_paths():
        cmd += ["-I", p]
    cmd += [os.path.join(CSRC, "ext.cpp"), "-o", EXT]
    for p in ce.library_paths():
        cmd += ["-L", p, f"-Wl,-rpath,{p}"]
    cmd += ["-L", LIB_DIR, "-Wl,-rpath,$ORIGIN/../lib", "-lovx_fdg",
            "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
    subprocess.check_call(cmd)
    return EXT


def build(force=False):
    build_lib(force)
    build_ext(force)
    return LIB, EXT


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_lib(force, verbose="-v" in sys.argv))
    print(build_ext(force))
