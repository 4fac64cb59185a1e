"""Build recipe for the reference's own CUDA path (measurement only).

Compiles the reference's four flexible-dual-grid CUDA sources
(``src/convert/mesh_to_flexible_dual_grid_gpu/{intersect_qef,face_qef,
boundary_qef,mesh_to_flexible_dual_grid}.cu``) unmodified, plus
``ref_gpu_binding.cpp``, into ``baseline/_ref/ref_fdg_gpu<EXT_SUFFIX>``.  The
reference builds these files with ``-O3 -std=c++17`` and no architecture flag
of its own (``setup.py:35-73``), i.e. generic code for the target GPU; here
that target is ``sm_100`` (B200).  nvcc's default FMA contraction is kept, as
in the reference build.

The source tree is read from ``$OVX_REFERENCE_ROOT``; without it nothing is
built and an existing build is kept.  ``baseline/_ref`` is git-ignored and
travels with the repository snapshot to the GPU machine.  The compile takes
about twenty minutes (the reference sources instantiate CUB and torch
templates heavily), so this recipe is run on its own rather than from
``__graft_entry__.build()``.
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
SO = os.path.join(OUT_DIR, "ref_fdg_gpu" + sysconfig.get_config_var("EXT_SUFFIX"))
SOURCES = ["intersect_qef.cu", "face_qef.cu", "boundary_qef.cu", "mesh_to_flexible_dual_grid.cu"]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build(force=False):
    """Returns the built module path, or None when neither the source tree nor a build exists."""
    root = os.environ.get("OVX_REFERENCE_ROOT")
    src_dir = os.path.join(root, "src") if root else None
    if not src_dir or not os.path.isdir(src_dir):
        return SO if os.path.exists(SO) else None
    fdg_dir = os.path.join(src_dir, "convert", "mesh_to_flexible_dual_grid_gpu")
    cu = [os.path.join(fdg_dir, s) for s in SOURCES]
    binding = os.path.join(HERE, "ref_gpu_binding.cpp")
    if not (force or _newer(SO, cu + [binding])):
        return SO
    import torch
    from torch.utils import cpp_extension as ce

    import tempfile

    os.makedirs(OUT_DIR, exist_ok=True)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    nvcc = os.path.join(cuda_home, "bin", "nvcc")
    defs = [f"-D_GLIBCXX_USE_CXX11_ABI={abi}", "-DTORCH_EXTENSION_NAME=ref_fdg_gpu", "-DTORCH_API_INCLUDE_EXTENSION_H"]
    incs = ["-I", src_dir, "-I", sysconfig.get_paths()["include"]]
    for p in ce.include_paths(device_type="cuda"):
        incs += ["-I", p]
    with tempfile.TemporaryDirectory() as tmp:
        objs = []
        for s in cu:
            o = os.path.join(tmp, os.path.basename(s) + ".o")
            # the flags torch's BuildExtension gives CUDA sources, with the reference's -O3 -std=c++17
            subprocess.check_call([nvcc, "-c", s, "-o", o, "-O3", "-std=c++17", "-gencode", "arch=compute_100,code=sm_100",
                                   "--expt-relaxed-constexpr", "-D__CUDA_NO_HALF_OPERATORS__", "-D__CUDA_NO_HALF_CONVERSIONS__",
                                   "-D__CUDA_NO_BFLOAT16_CONVERSIONS__", "-D__CUDA_NO_HALF2_OPERATORS__",
                                   "-Xcompiler", "-fPIC", "-w", *defs, *incs])
            objs.append(o)
        ob = os.path.join(tmp, "ref_gpu_binding.o")
        subprocess.check_call(["g++", "-c", binding, "-o", ob, "-O3", "-std=c++17", "-fPIC", "-w", *defs, *incs,
                               "-I", os.path.join(cuda_home, "include")])
        objs.append(ob)
        cmd = ["g++", "-shared", "-o", SO, *objs]
        for p in ce.library_paths(device_type="cuda"):
            cmd += ["-L", p, f"-Wl,-rpath,{p}"]
        cmd += ["-L", os.path.join(cuda_home, "lib64"), "-lcudart",
                "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
        subprocess.check_call(cmd)
    return SO


def load():
    """Imports the built module (None if it was never built)."""
    if not os.path.exists(SO):
        return None
    import importlib.util

    import torch  # noqa: F401  (the module links against torch)

    spec = importlib.util.spec_from_file_location("ref_fdg_gpu", SO)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
