// Binding for the reference's own GPU hashmap (src/hash/hash.cu, declared in
// src/hash/api.h, bound in the reference's src/ext.cpp:12-16), compiled from
// its source by oracle/build.py.  TEST INFRASTRUCTURE ONLY: it pins the CPU
// restatement of the two hashmap operations that
// o_voxel.convert.flexible_dual_grid_to_mesh calls
// (o_voxel/convert/flexible_dual_grid.py:430,437), which the golden fixture
// script runs the reference's own Python function with.
#include <torch/extension.h>
#include "hash/api.h"

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    m.def("hashmap_insert_3d_idx_as_val_cuda", &hashmap_insert_3d_idx_as_val_cuda);
    m.def("hashmap_lookup_3d_cuda", &hashmap_lookup_3d_cuda);
}
