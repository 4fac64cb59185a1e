"""Build recipe for the oracle (test infrastructure only).

Two artefacts:

* ``oracle/libfdg_oracle.so`` -- the plain-C restatement (``fdg_oracle.c``).
* ``oracle/_ref/fdg_ref<EXT_SUFFIX>`` -- the reference's own CPU implementation
  of the path, ``src/convert/flexible_dual_grid.cpp`` compiled unmodified from
  the reference source tree against the project's Eigen-API shim
  (``oracle/eigen_shim``; Eigen is an un-vendored submodule of the reference),
  plus ``ref_binding.cpp``.  Built only where the reference tree exists; the
  built file travels with the repository snapshot to machines without it.

Flags follow the reference's own build (``setup.py:65-67``: ``-O3 -std=c++17``,
no ``-march``), with ``-ffp-contract=off`` stated explicitly.
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree; without it nothing is rebuilt and existing builds are kept
REFERENCE_ROOT = os.environ.get("OVX_REFERENCE_ROOT", "")
ORACLE_SO = os.path.join(HERE, "libfdg_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "fdg_ref" + sysconfig.get_config_var("EXT_SUFFIX"))


def _ref_src(*parts):
    """Path of a file of the reference source tree, or None when OVX_REFERENCE_ROOT is unset."""
    return os.path.join(REFERENCE_ROOT, *parts) if REFERENCE_ROOT else None


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force=False):
    src = [os.path.join(HERE, "fdg_oracle.c"), os.path.join(HERE, "fdg_oracle_impl.h")]
    if force or _newer(ORACLE_SO, src):
        cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fPIC", "-shared", src[0], "-o", ORACLE_SO, "-lm"]
        subprocess.check_call(cmd)
    return ORACLE_SO


def build_ref(force=False):
    """Compile the reference CPU path; returns the .so path or None if the source is absent."""
    ref_cpp = _ref_src("src", "convert", "flexible_dual_grid.cpp")
    if not ref_cpp or not os.path.exists(ref_cpp):
        return REF_SO if os.path.exists(REF_SO) else None
    binding = os.path.join(HERE, "ref_binding.cpp")
    shim = os.path.join(HERE, "eigen_shim")
    if not (force or _newer(REF_SO, [ref_cpp, binding, os.path.join(shim, "Eigen", "Dense")])):
        return REF_SO
    import torch
    from torch.utils import cpp_extension as ce

    os.makedirs(REF_DIR, exist_ok=True)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O3", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
           "-w", "-fext-numeric-literals",
           f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-DTORCH_EXTENSION_NAME=fdg_ref", "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-I", shim, "-I", os.path.dirname(ref_cpp), "-I", sysconfig.get_paths()["include"]]
    for p in ce.include_paths():
        cmd += ["-I", p]
    cmd += [ref_cpp, binding, "-o", REF_SO]
    for p in ce.library_paths():
        cmd += ["-L", p, f"-Wl,-rpath,{p}"]
    cmd += ["-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python"]
    subprocess.check_call(cmd)
    return REF_SO


REF_ZORDER_SO = os.path.join(REF_DIR, "zorder_ref.so")


def build_ref_zorder(force=False):
    """Compile the reference's z-order source (src/serialize/z_order.cu; its
    CPU functions are what the binding calls) into oracle/_ref; returns the .so
    path or None if the source is absent."""
    src = _ref_src("src", "serialize", "z_order.cu")
    if not src or not os.path.exists(src):
        return REF_ZORDER_SO if os.path.exists(REF_ZORDER_SO) else None
    binding = os.path.join(HERE, "ref_zorder_binding.cu")
    if not (force or _newer(REF_ZORDER_SO, [src, binding])):
        return REF_ZORDER_SO
    os.makedirs(REF_DIR, exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.dirname(src), src, binding, "-o", REF_ZORDER_SO]
    subprocess.check_call(cmd)
    return REF_ZORDER_SO


REF_HILBERT_SO = os.path.join(REF_DIR, "hilbert_ref.so")


def build_ref_hilbert(force=False):
    """Compile the reference's Hilbert source (src/serialize/hilbert.cu; its CPU
    functions are what the binding calls) into oracle/_ref; returns the .so path
    or None if the source is absent."""
    src = _ref_src("src", "serialize", "hilbert.cu")
    if not src or not os.path.exists(src):
        return REF_HILBERT_SO if os.path.exists(REF_HILBERT_SO) else None
    binding = os.path.join(HERE, "ref_hilbert_binding.cu")
    if not (force or _newer(REF_HILBERT_SO, [src, binding])):
        return REF_HILBERT_SO
    os.makedirs(REF_DIR, exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    cmd = [nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.dirname(src), src, binding, "-o", REF_HILBERT_SO]
    subprocess.check_call(cmd)
    return REF_HILBERT_SO


REF_HASH_SO = os.path.join(REF_DIR, "hash_ref" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_ref_hash(force=False):
    """Compile the reference's GPU hashmap (src/hash/hash.cu) with
    ref_hash_binding.cpp into oracle/_ref, as a torch extension for sm_100
    (the reference's generic build, setup.py:35-73); returns the .so path or
    None if neither the source nor a build exists."""
    src = _ref_src("src", "hash", "hash.cu")
    if not src or not os.path.exists(src):
        return REF_HASH_SO if os.path.exists(REF_HASH_SO) else None
    binding = os.path.join(HERE, "ref_hash_binding.cpp")
    if not (force or _newer(REF_HASH_SO, [src, binding])):
        return REF_HASH_SO
    import tempfile

    import torch
    from torch.utils import cpp_extension as ce

    os.makedirs(REF_DIR, exist_ok=True)
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    defs = [f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-DTORCH_EXTENSION_NAME=hash_ref", "-DTORCH_API_INCLUDE_EXTENSION_H"]
    incs = ["-I", os.path.join(REFERENCE_ROOT, "src"), "-I", sysconfig.get_paths()["include"],
            "-I", os.path.join(cuda_home, "include")]
    for p in ce.include_paths(device_type="cuda"):
        incs += ["-I", p]
    with tempfile.TemporaryDirectory() as tmp:
        o1, o2 = os.path.join(tmp, "hash.o"), os.path.join(tmp, "binding.o")
        subprocess.check_call([os.path.join(cuda_home, "bin", "nvcc"), "-c", src, "-o", o1, "-O3", "-std=c++17",
                               "-gencode", "arch=compute_100,code=sm_100", "--expt-relaxed-constexpr",
                               "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
                               "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
                               "-Xcompiler", "-fPIC", "-w", *defs, *incs])
        subprocess.check_call(["g++", "-c", binding, "-o", o2, "-O3", "-std=c++17", "-fPIC", "-w", *defs, *incs])
        cmd = ["g++", "-shared", "-o", REF_HASH_SO, o1, o2]
        for p in ce.library_paths(device_type="cuda"):
            cmd += ["-L", p, f"-Wl,-rpath,{p}"]
        cmd += ["-L", os.path.join(cuda_home, "lib64"), "-lcudart",
                "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
        subprocess.check_call(cmd)
    return REF_HASH_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
    print(build_ref_zorder(force="--force" in sys.argv))
    print(build_ref_hilbert(force="--force" in sys.argv))
    print(build_ref_hash(force="--force" in sys.argv))
