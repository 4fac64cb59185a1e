// Minimal binding of the reference's own CUDA implementation of the path
// (o_voxel._C.mesh_to_flexible_dual_grid_cuda / intersect_occ_cuda, bound in
// the reference's src/ext.cpp:19,21 and declared in src/convert/api.h:53-174),
// compiled from the reference's sources by baseline/build_ref_gpu.py.  Only the
// two conversion operators are bound: the reference's own src/ext.cpp also
// binds its Eigen-based CPU code and unrelated subsystems.  Used by bench.py to
// time the reference GPU path on the same B200 as this library.
#include <torch/extension.h>
#include "convert/api.h"

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.def("mesh_to_flexible_dual_grid_cuda", &o_voxel::fdg::mesh_to_flexible_dual_grid_cuda,
          py::call_guard<py::gil_scoped_release>());
    m.def("intersect_occ_cuda", &o_voxel::fdg::intersect_occ_cuda, py::call_guard<py::gil_scoped_release>());
}
