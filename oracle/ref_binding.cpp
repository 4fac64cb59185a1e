// Binding for the reference's own CPU implementation of the path, compiled
// from its source (src/convert/flexible_dual_grid.cpp) against the Eigen-API
// shim in oracle/eigen_shim.  TEST INFRASTRUCTURE ONLY: used to pin the C
// oracle and as the timed CPU reference arm of the benchmark.
#include <torch/extension.h>
#include "api.h" // reference declarations: src/convert/api.h:31-51

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.def("mesh_to_flexible_dual_grid_cpu", &mesh_to_flexible_dual_grid_cpu, py::call_guard<py::gil_scoped_release>());
    m.def("intersect_occ_cpu", &intersect_occ_cpu, py::call_guard<py::gil_scoped_release>());
}
