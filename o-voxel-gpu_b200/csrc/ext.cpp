// ext.cpp -- torch extension `o_voxel._C` for the B200 flexible-dual-grid
// library.  Mirrors the reference binding (src/ext.cpp:18-21) for this path:
//
//   mesh_to_flexible_dual_grid_cuda(vertices, faces, voxel_size, grid_range,
//       face_weight, boundary_weight, regularization_weight)
//       -> (voxels int32[N,3], dual_vertices float32[N,3], intersected bool[N,3])
//       reference: src/convert/api.h:164-172
//   intersect_occ_cuda(triangles, voxel_size, grid_range) -> int32[N,3]
//       reference: src/convert/api.h:63-66
//
// plus `mesh_to_flexible_dual_grid_cuda_ex`, which takes unshifted vertices,
// the aabb origin and int32 or int64 faces so the wrapper does not need the
// extra cast and shift passes over the inputs, and
// `mesh_to_flexible_dual_grid_cuda_batch`, which converts a list of meshes
// (each with its own grid) through the library's batched conversion: every
// kernel runs once over a group of meshes, with one host synchronisation per
// group; groups bound the workspace by an estimate of their records.
//
// All compute goes through the C ABI in include/ovx_fdg.h (libovx_fdg.so).
// Setting OVX_FDG_CHECK in the environment makes every call wait for its
// device-side consistency checks (ovx_fdg_sync_status) and raise on failure.
// Outputs come from torch's caching allocator on the input's device, work runs
// on torch's current stream, and the GIL is released during the call, as in
// the reference.  Errors raise RuntimeError (TORCH_CHECK), as in the reference.
#include <torch/extension.h>
#include <ATen/cuda/CUDAContext.h>
#include <c10/cuda/CUDAGuard.h>

#include <c10/cuda/CUDAStream.h>

#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "ovx_fdg.h"

namespace
{

struct DeviceContext
{
    ovx_fdg_context *ctx = nullptr;
    std::mutex mu;
    ~DeviceContext()
    {
        if (ctx)
            ovx_fdg_context_destroy(ctx);
    }
};

DeviceContext &context_for(int device)
{
    static std::mutex map_mu;
    static std::map<int, std::unique_ptr<DeviceContext>> contexts;
    std::lock_guard<std::mutex> lock(map_mu);
    auto &slot = contexts[device];
    if (!slot)
    {
        slot = std::make_unique<DeviceContext>();
        const int rc = ovx_fdg_context_create(device, &slot->ctx);
        TORCH_CHECK(rc == OVX_FDG_OK, "ovx_fdg_context_create failed: ", ovx_fdg_status_string(rc));
    }
    return *slot;
}

void check(int rc, ovx_fdg_context *ctx, const char *what)
{
    TORCH_CHECK(rc == OVX_FDG_OK, what, " failed (", ovx_fdg_status_string(rc), "): ", ovx_fdg_last_error(ctx));
}

ovx_fdg_grid make_grid(const std::vector<float> &voxel_size, const std::vector<int64_t> &grid_range)
{
    TORCH_CHECK(voxel_size.size() == 3, "voxel_size must have 3 elements");
    TORCH_CHECK(grid_range.size() == 6, "grid_range must have 6 elements");
    ovx_fdg_grid g;
    for (int a = 0; a < 3; ++a)
    {
        g.voxel_size[a] = voxel_size[a];
        g.grid_min[a] = static_cast<int32_t>(grid_range[a]);
        g.grid_max[a] = static_cast<int32_t>(grid_range[3 + a]);
    }
    return g;
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> run_fdg(const torch::Tensor &vertices, const torch::Tensor &faces,
                                                                 const float *origin, const std::vector<float> &voxel_size,
                                                                 const std::vector<int64_t> &grid_range, float face_weight,
                                                                 float boundary_weight, float regularization_weight, int64_t order,
                                                                 int64_t precision, double route_tolerance)
{
    TORCH_CHECK(vertices.is_cuda(), "vertices must be a CUDA tensor");
    TORCH_CHECK(faces.is_cuda(), "faces must be a CUDA tensor");
    TORCH_CHECK(vertices.device() == faces.device(), "vertices and faces must be on the same device");
    TORCH_CHECK(vertices.scalar_type() == torch::kFloat32, "vertices must be float32");
    TORCH_CHECK(faces.scalar_type() == torch::kInt32 || faces.scalar_type() == torch::kInt64, "faces must be int32 or int64");
    TORCH_CHECK(vertices.dim() == 2 && vertices.size(1) == 3, "vertices must be [V,3]");
    TORCH_CHECK(faces.dim() == 2 && faces.size(1) == 3, "faces must be [F,3]");
    auto v = vertices.contiguous();
    auto f = faces.contiguous();
    const ovx_fdg_grid grid = make_grid(voxel_size, grid_range);
    const c10::cuda::CUDAGuard guard(v.device());
    const int device = v.get_device();
    cudaStream_t stream = at::cuda::getCurrentCUDAStream(device).stream();
    DeviceContext &dc = context_for(device);
    std::lock_guard<std::mutex> lock(dc.mu);
    check(ovx_fdg_set_output_order(dc.ctx, (int)order), dc.ctx, "mesh_to_flexible_dual_grid (order)");
    check(ovx_fdg_set_precision(dc.ctx, (int)precision, (float)route_tolerance), dc.ctx, "mesh_to_flexible_dual_grid (precision)");
    int64_t n = 0;
    check(ovx_fdg_begin(dc.ctx, stream, v.data_ptr<float>(), v.size(0), f.numel() ? f.data_ptr() : nullptr,
                        f.scalar_type() == torch::kInt64 ? 8 : 4, f.size(0), origin, &grid, face_weight, boundary_weight,
                        regularization_weight, &n),
          dc.ctx, "mesh_to_flexible_dual_grid (occupancy)");
    auto opts = torch::TensorOptions().device(v.device());
    auto vox = torch::empty({n, 3}, opts.dtype(torch::kInt32));
    auto dual = torch::empty({n, 3}, opts.dtype(torch::kFloat32));
    auto inter = torch::empty({n, 3}, opts.dtype(torch::kBool));
    check(ovx_fdg_finish(dc.ctx, stream, n ? vox.data_ptr<int32_t>() : nullptr, n ? dual.data_ptr<float>() : nullptr,
                         n ? reinterpret_cast<uint8_t *>(inter.data_ptr<bool>()) : nullptr),
          dc.ctx, "mesh_to_flexible_dual_grid (quadrics)");
    static const bool sync_check = std::getenv("OVX_FDG_CHECK") != nullptr;
    if (sync_check)
        check(ovx_fdg_sync_status(dc.ctx, stream), dc.ctx, "mesh_to_flexible_dual_grid (device checks)");
    return std::make_tuple(vox, dual, inter);
}

// Context of the batched path on a device, kept for the life of the process
// like the single-mesh context.
DeviceContext &batch_context(int device)
{
    static std::mutex map_mu;
    static std::map<int, std::unique_ptr<DeviceContext>> contexts;
    std::lock_guard<std::mutex> lock(map_mu);
    auto &slot = contexts[device];
    if (!slot)
    {
        slot = std::make_unique<DeviceContext>();
        const int rc = ovx_fdg_context_create(device, &slot->ctx);
        TORCH_CHECK(rc == OVX_FDG_OK, "ovx_fdg_context_create failed: ", ovx_fdg_status_string(rc));
    }
    return *slot;
}

// Records a mesh is expected to produce, for sizing batch groups: about eight
// per unit of grid face area and three per triangle (the measured mixture of
// surface-bound and face-bound meshes stays below this on average).
int64_t estimated_records(const ovx_fdg_grid &g, int64_t faces)
{
    const int64_t x = g.grid_max[0] - g.grid_min[0], y = g.grid_max[1] - g.grid_min[1], z = g.grid_max[2] - g.grid_min[2];
    return 8 * (x * y + y * z + z * x) + 3 * faces;
}

} // namespace

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> mesh_to_flexible_dual_grid_cuda(
    const torch::Tensor &vertices, const torch::Tensor &faces, const std::vector<float> &voxel_size,
    const std::vector<int64_t> &grid_range, float face_weight, float boundary_weight, float regularization_weight,
    int64_t order, int64_t precision, double route_tolerance)
{
    return run_fdg(vertices, faces, nullptr, voxel_size, grid_range, face_weight, boundary_weight, regularization_weight, order,
                   precision, route_tolerance);
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> mesh_to_flexible_dual_grid_cuda_ex(
    const torch::Tensor &vertices, const torch::Tensor &faces, const std::vector<float> &origin,
    const std::vector<float> &voxel_size, const std::vector<int64_t> &grid_range, float face_weight, float boundary_weight,
    float regularization_weight, int64_t order, int64_t precision, double route_tolerance)
{
    TORCH_CHECK(origin.size() == 3, "origin must have 3 elements");
    const float o[3] = {origin[0], origin[1], origin[2]};
    return run_fdg(vertices, faces, o, voxel_size, grid_range, face_weight, boundary_weight, regularization_weight, order,
                   precision, route_tolerance);
}

torch::Tensor intersect_occ_cuda(const torch::Tensor &triangles, const std::vector<float> &voxel_size,
                                 const std::vector<int64_t> &grid_range, int64_t order)
{
    TORCH_CHECK(triangles.is_cuda(), "triangles must be a CUDA tensor");
    TORCH_CHECK(triangles.scalar_type() == torch::kFloat32, "triangles must be float32");
    TORCH_CHECK(triangles.dim() == 3 && triangles.size(1) == 3 && triangles.size(2) == 3, "triangles must be [T,3,3]");
    auto t = triangles.contiguous();
    const ovx_fdg_grid grid = make_grid(voxel_size, grid_range);
    const c10::cuda::CUDAGuard guard(t.device());
    const int device = t.get_device();
    cudaStream_t stream = at::cuda::getCurrentCUDAStream(device).stream();
    DeviceContext &dc = context_for(device);
    std::lock_guard<std::mutex> lock(dc.mu);
    check(ovx_fdg_set_output_order(dc.ctx, (int)order), dc.ctx, "intersect_occ (order)");
    int64_t n = 0;
    check(ovx_fdg_occupancy_begin(dc.ctx, stream, t.numel() ? t.data_ptr<float>() : nullptr, t.size(0), &grid, &n), dc.ctx,
          "intersect_occ");
    auto vox = torch::empty({n, 3}, torch::TensorOptions().device(t.device()).dtype(torch::kInt32));
    check(ovx_fdg_occupancy_finish(dc.ctx, stream, n ? vox.data_ptr<int32_t>() : nullptr), dc.ctx, "intersect_occ");
    return vox;
}

std::vector<std::tuple<torch::Tensor, torch::Tensor, torch::Tensor>> mesh_to_flexible_dual_grid_cuda_batch(
    const std::vector<torch::Tensor> &vertices, const std::vector<torch::Tensor> &faces,
    const std::vector<std::vector<float>> &origins, const std::vector<std::vector<float>> &voxel_sizes,
    const std::vector<std::vector<int64_t>> &grid_ranges, float face_weight, float boundary_weight,
    float regularization_weight, int64_t max_group_records, int64_t order, int64_t precision, double route_tolerance)
{
    const size_t n = vertices.size();
    TORCH_CHECK(faces.size() == n && origins.size() == n && voxel_sizes.size() == n && grid_ranges.size() == n,
                "mesh_to_flexible_dual_grid_batch: per-mesh argument lists differ in length");
    std::vector<std::tuple<torch::Tensor, torch::Tensor, torch::Tensor>> out(n);
    if (n == 0)
        return out;
    const c10::Device dev = vertices[0].device();
    std::vector<torch::Tensor> vs(n), fs(n);
    std::vector<ovx_fdg_mesh> meshes(n);
    for (size_t i = 0; i < n; ++i)
    {
        TORCH_CHECK(vertices[i].is_cuda() && faces[i].is_cuda(), "mesh ", i, ": vertices and faces must be CUDA tensors");
        TORCH_CHECK(vertices[i].device() == dev && faces[i].device() == dev, "mesh ", i, ": all meshes must be on one device");
        TORCH_CHECK(vertices[i].scalar_type() == torch::kFloat32, "mesh ", i, ": vertices must be float32");
        TORCH_CHECK(faces[i].scalar_type() == torch::kInt32 || faces[i].scalar_type() == torch::kInt64,
                    "mesh ", i, ": faces must be int32 or int64");
        TORCH_CHECK(vertices[i].dim() == 2 && vertices[i].size(1) == 3, "mesh ", i, ": vertices must be [V,3]");
        TORCH_CHECK(faces[i].dim() == 2 && faces[i].size(1) == 3, "mesh ", i, ": faces must be [F,3]");
        TORCH_CHECK(origins[i].size() == 3, "mesh ", i, ": origin must have 3 elements");
        vs[i] = vertices[i].contiguous();
        fs[i] = faces[i].contiguous();
        ovx_fdg_mesh &m = meshes[i];
        m.vertices = vs[i].numel() ? vs[i].data_ptr<float>() : nullptr;
        m.num_vertices = vs[i].size(0);
        m.faces = fs[i].numel() ? fs[i].data_ptr() : nullptr;
        m.face_index_bytes = fs[i].scalar_type() == torch::kInt64 ? 8 : 4;
        m.num_faces = fs[i].size(0);
        for (int a = 0; a < 3; ++a)
            m.origin[a] = origins[i][a];
        m.grid = make_grid(voxel_sizes[i], grid_ranges[i]);
    }
    const c10::cuda::CUDAGuard guard(dev);
    const int device = dev.index();
    cudaStream_t stream = at::cuda::getCurrentCUDAStream(device).stream();
    DeviceContext &dc = batch_context(device);
    std::lock_guard<std::mutex> lock(dc.mu);
    check(ovx_fdg_set_output_order(dc.ctx, (int)order), dc.ctx, "mesh_to_flexible_dual_grid_batch (order)");
    check(ovx_fdg_set_precision(dc.ctx, (int)precision, (float)route_tolerance), dc.ctx,
          "mesh_to_flexible_dual_grid_batch (precision)");
    static const bool sync_check = std::getenv("OVX_FDG_CHECK") != nullptr;
    auto opts = torch::TensorOptions().device(dev);
    // groups of consecutive meshes whose expected records stay within the
    // budget: one conversion (one host synchronisation) per group
    size_t first = 0;
    while (first < n)
    {
        size_t last = first + 1;
        int64_t est = estimated_records(meshes[first].grid, meshes[first].num_faces);
        while (last < n)
        {
            const int64_t e = estimated_records(meshes[last].grid, meshes[last].num_faces);
            if (max_group_records > 0 && est + e > max_group_records)
                break;
            est += e;
            ++last;
        }
        const int32_t gm = (int32_t)(last - first);
        std::vector<int64_t> nvox((size_t)gm);
        int64_t total = 0;
        check(ovx_fdg_begin_batch(dc.ctx, stream, meshes.data() + first, gm, face_weight, boundary_weight, regularization_weight,
                                  nvox.data(), &total),
              dc.ctx, "mesh_to_flexible_dual_grid_batch (occupancy)");
        auto vox = torch::empty({total, 3}, opts.dtype(torch::kInt32));
        auto dual = torch::empty({total, 3}, opts.dtype(torch::kFloat32));
        auto inter = torch::empty({total, 3}, opts.dtype(torch::kBool));
        check(ovx_fdg_finish_batch(dc.ctx, stream, total ? vox.data_ptr<int32_t>() : nullptr, total ? dual.data_ptr<float>() : nullptr,
                                   total ? reinterpret_cast<uint8_t *>(inter.data_ptr<bool>()) : nullptr),
              dc.ctx, "mesh_to_flexible_dual_grid_batch (quadrics)");
        if (sync_check)
            check(ovx_fdg_sync_status(dc.ctx, stream), dc.ctx, "mesh_to_flexible_dual_grid_batch (device checks)");
        int64_t row = 0;
        for (int32_t k = 0; k < gm; ++k)
        {
            const int64_t r = nvox[(size_t)k];
            out[first + (size_t)k] = std::make_tuple(vox.narrow(0, row, r), dual.narrow(0, row, r), inter.narrow(0, row, r));
            row += r;
        }
        first = last;
    }
    return out;
}

// Work shapes (ovx_fdg_tuning, in field order) of the device's single-mesh and
// batch contexts; an empty list restores the defaults.
void set_tuning_cuda(int64_t device, const std::vector<int64_t> &values)
{
    TORCH_CHECK(values.empty() || values.size() == 5, "set_tuning: 5 values (or none) expected");
    ovx_fdg_tuning t{};
    if (!values.empty())
    {
        t.unit_cells = (int32_t)values[0];
        t.warp_scan_cells = (int32_t)values[1];
        t.inline_face_bricks = (int32_t)values[2];
        t.dense_candidates = (int32_t)values[3];
        t.long_walk = (int32_t)values[4];
    }
    for (DeviceContext *dc : {&context_for((int)device), &batch_context((int)device)})
    {
        std::lock_guard<std::mutex> lock(dc->mu);
        check(ovx_fdg_set_tuning(dc->ctx, values.empty() ? nullptr : &t), dc->ctx, "set_tuning");
    }
}

// flexible dual grid -> mesh (reference o_voxel/convert/flexible_dual_grid.py:332-477)
std::tuple<torch::Tensor, torch::Tensor> flexible_dual_grid_to_mesh_cuda(
    const torch::Tensor &coords, const torch::Tensor &dual_vertices, const torch::Tensor &intersected,
    const c10::optional<torch::Tensor> &split_weight, const std::vector<int64_t> &grid_size,
    const std::vector<float> &voxel_size, const std::vector<float> &aabb_min, bool train)
{
    TORCH_CHECK(coords.is_cuda() && dual_vertices.is_cuda() && intersected.is_cuda(), "flexible_dual_grid_to_mesh: CUDA tensors expected");
    TORCH_CHECK(coords.dim() == 2 && coords.size(1) == 3, "coords must be [N,3]");
    const int64_t n = coords.size(0);
    TORCH_CHECK(dual_vertices.dim() == 2 && dual_vertices.size(0) == n && dual_vertices.size(1) == 3, "dual_vertices must be [N,3]");
    TORCH_CHECK(intersected.numel() == 3 * n, "intersected must have N x 3 entries");
    TORCH_CHECK(grid_size.size() == 3 && voxel_size.size() == 3 && aabb_min.size() == 3, "grid_size, voxel_size, aabb_min need 3 values");
    const c10::cuda::CUDAGuard guard(coords.device());
    const int device = coords.get_device();
    auto c = coords.to(torch::kInt32).contiguous();
    auto d = dual_vertices.to(torch::kFloat32).contiguous();
    auto f = intersected.to(torch::kUInt8).contiguous();
    torch::Tensor w;
    if (split_weight.has_value() && split_weight->defined())
    {
        w = split_weight->to(torch::kFloat32).contiguous();
        TORCH_CHECK(w.numel() == n, "split_weight must have one value per voxel");
    }
    TORCH_CHECK(!train || w.defined(), "split_weight must be provided in training mode");
    static std::mutex map_mu;
    static std::map<int, ovx_fdg_mesh_context *> contexts;
    static std::map<int, std::unique_ptr<std::mutex>> locks;
    ovx_fdg_mesh_context *ctx = nullptr;
    std::mutex *mu = nullptr;
    {
        std::lock_guard<std::mutex> lock(map_mu);
        auto &slot = contexts[device];
        if (!slot)
        {
            const int rc = ovx_fdg_mesh_context_create(device, &slot);
            TORCH_CHECK(rc == OVX_FDG_OK, "ovx_fdg_mesh_context_create failed: ", ovx_fdg_status_string(rc));
            locks[device] = std::make_unique<std::mutex>();
        }
        ctx = slot;
        mu = locks[device].get();
    }
    std::lock_guard<std::mutex> lock(*mu);
    cudaStream_t stream = at::cuda::getCurrentCUDAStream(device).stream();
    const int32_t gs[3] = {(int32_t)grid_size[0], (int32_t)grid_size[1], (int32_t)grid_size[2]};
    const float vs[3] = {voxel_size[0], voxel_size[1], voxel_size[2]};
    const float am[3] = {aabb_min[0], aabb_min[1], aabb_min[2]};
    int64_t nv = 0, nt = 0;
    int rc = ovx_fdg_to_mesh_begin(ctx, stream, n ? c.data_ptr<int32_t>() : nullptr, n ? d.data_ptr<float>() : nullptr,
                                   n ? f.data_ptr<uint8_t>() : nullptr, w.defined() ? w.data_ptr<float>() : nullptr, n, gs, vs,
                                   am, train ? 1 : 0, &nv, &nt);
    TORCH_CHECK(rc == OVX_FDG_OK, "flexible_dual_grid_to_mesh failed (", ovx_fdg_status_string(rc), "): ", ovx_fdg_mesh_last_error(ctx));
    auto opts = torch::TensorOptions().device(coords.device());
    auto verts = torch::empty({nv, 3}, opts.dtype(torch::kFloat32));
    auto tris = torch::empty({nt, 3}, opts.dtype(torch::kInt32));
    rc = ovx_fdg_to_mesh_finish(ctx, stream, nv ? verts.data_ptr<float>() : nullptr, nt ? tris.data_ptr<int32_t>() : nullptr);
    TORCH_CHECK(rc == OVX_FDG_OK, "flexible_dual_grid_to_mesh failed (", ovx_fdg_status_string(rc), "): ", ovx_fdg_mesh_last_error(ctx));
    return std::make_tuple(verts, tris);
}

// .vxz attribute packing (reference examples/mesh2ovox.py:51-54)
std::tuple<torch::Tensor, torch::Tensor> pack_flexible_dual_grid_cuda(const torch::Tensor &voxels, const torch::Tensor &dual,
                                                                     const torch::Tensor &intersected, const std::vector<float> &resolution)
{
    TORCH_CHECK(voxels.is_cuda() && dual.is_cuda() && intersected.is_cuda(), "pack_flexible_dual_grid: CUDA tensors expected");
    TORCH_CHECK(resolution.size() == 3, "resolution must have 3 values");
    const int64_t n = voxels.size(0);
    TORCH_CHECK(dual.numel() == 3 * n && intersected.numel() == 3 * n, "inputs must all have N x 3 entries");
    const c10::cuda::CUDAGuard guard(voxels.device());
    auto v = voxels.to(torch::kInt32).contiguous();
    auto d = dual.to(torch::kFloat32).contiguous();
    auto f = intersected.to(torch::kUInt8).contiguous();
    auto opts = torch::TensorOptions().device(voxels.device()).dtype(torch::kUInt8);
    auto du = torch::empty({n, 3}, opts);
    auto fu = torch::empty({n, 1}, opts);
    const float r[3] = {resolution[0], resolution[1], resolution[2]};
    const int rc = ovx_fdg_pack(at::cuda::getCurrentCUDAStream(voxels.get_device()).stream(), n ? v.data_ptr<int32_t>() : nullptr,
                                n ? d.data_ptr<float>() : nullptr, n ? f.data_ptr<uint8_t>() : nullptr, n, r,
                                n ? du.data_ptr<uint8_t>() : nullptr, n ? fu.data_ptr<uint8_t>() : nullptr);
    TORCH_CHECK(rc == OVX_FDG_OK, "pack_flexible_dual_grid failed: ", ovx_fdg_status_string(rc));
    return std::make_tuple(du, fu);
}

// o_voxel.serialize codes (reference: src/ext.cpp:28-31, src/serialize/api.cu): z-order and Hilbert
using EncodeFn = int (*)(void *, const int32_t *, const int32_t *, const int32_t *, int64_t, int32_t *);
using DecodeFn = int (*)(void *, const int32_t *, int64_t, int32_t *, int32_t *, int32_t *);

torch::Tensor encode_codes(EncodeFn fn, const char *name, const torch::Tensor &x, const torch::Tensor &y, const torch::Tensor &z)
{
    TORCH_CHECK(x.is_cuda() && y.is_cuda() && z.is_cuda(), name, ": CUDA tensors expected");
    TORCH_CHECK(x.numel() == y.numel() && x.numel() == z.numel(), name, ": x, y, z differ in length");
    const c10::cuda::CUDAGuard guard(x.device());
    auto xi = x.to(torch::kInt32).contiguous(), yi = y.to(torch::kInt32).contiguous(), zi = z.to(torch::kInt32).contiguous();
    auto codes = torch::empty_like(xi);
    const int rc = fn(at::cuda::getCurrentCUDAStream(x.get_device()).stream(), xi.data_ptr<int32_t>(), yi.data_ptr<int32_t>(),
                      zi.data_ptr<int32_t>(), xi.numel(), codes.data_ptr<int32_t>());
    TORCH_CHECK(rc == OVX_FDG_OK, name, " failed: ", ovx_fdg_status_string(rc));
    return codes;
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> decode_codes(DecodeFn fn, const char *name, const torch::Tensor &codes)
{
    TORCH_CHECK(codes.is_cuda(), name, ": CUDA tensor expected");
    const c10::cuda::CUDAGuard guard(codes.device());
    auto c = codes.to(torch::kInt32).contiguous();
    auto x = torch::empty_like(c), y = torch::empty_like(c), z = torch::empty_like(c);
    const int rc = fn(at::cuda::getCurrentCUDAStream(codes.get_device()).stream(), c.data_ptr<int32_t>(), c.numel(),
                      x.data_ptr<int32_t>(), y.data_ptr<int32_t>(), z.data_ptr<int32_t>());
    TORCH_CHECK(rc == OVX_FDG_OK, name, " failed: ", ovx_fdg_status_string(rc));
    return std::make_tuple(x, y, z);
}

torch::Tensor z_order_encode_cuda(const torch::Tensor &x, const torch::Tensor &y, const torch::Tensor &z)
{
    return encode_codes(ovx_z_order_encode, "z_order_encode_cuda", x, y, z);
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> z_order_decode_cuda(const torch::Tensor &codes)
{
    return decode_codes(ovx_z_order_decode, "z_order_decode_cuda", codes);
}

torch::Tensor hilbert_encode_cuda(const torch::Tensor &x, const torch::Tensor &y, const torch::Tensor &z)
{
    return encode_codes(ovx_hilbert_encode, "hilbert_encode_cuda", x, y, z);
}

std::tuple<torch::Tensor, torch::Tensor, torch::Tensor> hilbert_decode_cuda(const torch::Tensor &codes)
{
    return decode_codes(ovx_hilbert_decode, "hilbert_decode_cuda", codes);
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    // `order` (0: brick order, 1: z-order) is this library's addition; the
    // first seven arguments are the reference operator's
    m.def("mesh_to_flexible_dual_grid_cuda", &mesh_to_flexible_dual_grid_cuda, py::arg("vertices"), py::arg("faces"),
          py::arg("voxel_size"), py::arg("grid_range"), py::arg("face_weight"), py::arg("boundary_weight"),
          py::arg("regularization_weight"), py::arg("order") = 0, py::arg("precision") = 0, py::arg("route_tolerance") = 1e-3,
          py::call_guard<py::gil_scoped_release>());
    m.def("mesh_to_flexible_dual_grid_cuda_ex", &mesh_to_flexible_dual_grid_cuda_ex, py::arg("vertices"), py::arg("faces"),
          py::arg("origin"), py::arg("voxel_size"), py::arg("grid_range"), py::arg("face_weight"),
          py::arg("boundary_weight"), py::arg("regularization_weight"), py::arg("order") = 0, py::arg("precision") = 0,
          py::arg("route_tolerance") = 1e-3, py::call_guard<py::gil_scoped_release>());
    m.def("intersect_occ_cuda", &intersect_occ_cuda, py::arg("triangles"), py::arg("voxel_size"), py::arg("grid_range"),
          py::arg("order") = 0, py::call_guard<py::gil_scoped_release>());
    m.def("mesh_to_flexible_dual_grid_cuda_batch", &mesh_to_flexible_dual_grid_cuda_batch, py::arg("vertices"),
          py::arg("faces"), py::arg("origins"), py::arg("voxel_sizes"), py::arg("grid_ranges"), py::arg("face_weight"),
          py::arg("boundary_weight"), py::arg("regularization_weight"), py::arg("max_group_records"), py::arg("order") = 0,
          py::arg("precision") = 0, py::arg("route_tolerance") = 1e-3, py::call_guard<py::gil_scoped_release>());
    m.def("set_tuning_cuda", &set_tuning_cuda, py::arg("device"), py::arg("values"), py::call_guard<py::gil_scoped_release>());
    m.def("z_order_encode_cuda", &z_order_encode_cuda, py::call_guard<py::gil_scoped_release>());
    m.def("flexible_dual_grid_to_mesh_cuda", &flexible_dual_grid_to_mesh_cuda, py::call_guard<py::gil_scoped_release>());
    m.def("pack_flexible_dual_grid_cuda", &pack_flexible_dual_grid_cuda, py::call_guard<py::gil_scoped_release>());
    m.def("z_order_decode_cuda", &z_order_decode_cuda, py::call_guard<py::gil_scoped_release>());
    m.def("hilbert_encode_cuda", &hilbert_encode_cuda, py::call_guard<py::gil_scoped_release>());
    m.def("hilbert_decode_cuda", &hilbert_decode_cuda, py::call_guard<py::gil_scoped_release>());
}
