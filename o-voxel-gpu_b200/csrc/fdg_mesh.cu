// fdg_mesh.cu -- flexible dual grid -> triangle mesh (the inverse path of the
// conversion), behind the C ABI in include/ovx_fdg.h.
//
// Follows o_voxel.convert.flexible_dual_grid_to_mesh
// (o_voxel/convert/flexible_dual_grid.py:332-477):
//   * active voxels are found by their flat key x*gy*gz + y*gz + z in a hash
//     table, as the reference's hashmap does (src/hash/hash.cu:366-420,
//     269-300); a neighbour outside [0, grid) on any axis is not looked up and
//     counts as absent, as in the reference's lookup kernel (hash.cu:283-286);
//   * every intersected edge (voxel, axis) whose four surrounding voxels are
//     all active gives one quad, in (voxel, axis) order;
//   * quads are split into two triangles by the larger normal alignment, or
//     by the split weights; in training mode a weighted middle vertex is added
//     and each quad becomes four triangles;
//   * vertex positions are (coords + dual) * voxel_size + aabb_min.
//
// Layout: hash keys u64 (empty = ~0), values u32, capacity a power of two of
// at least 2N; per (voxel, axis) the four neighbour indices of a candidate
// quad (or an invalid marker) and its compaction flag.
#include "ovx_fdg.h"

#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace
{

constexpr unsigned long long kEmptyKey = ~0ull;
constexpr uint32_t kNoVoxel = 0xffffffffu;
constexpr int kThreads = 256;

inline unsigned blocks_for(long long n, int threads)
{
    return (unsigned)((n + threads - 1) / threads);
}

// 64-bit finaliser (a bijective mix), then masked to the table size.
__device__ __forceinline__ unsigned long long mix64(unsigned long long k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

struct MeshGrid
{
    long long gx, gy, gz;
    float vs[3];
    float amin[3];
};

__device__ __forceinline__ unsigned long long flat_key(const MeshGrid &g, long long x, long long y, long long z)
{
    return (unsigned long long)(x * g.gy * g.gz + y * g.gz + z);
}

__global__ void mesh_hash_insert(const int32_t *__restrict__ coords, long long n, MeshGrid g, unsigned long long *__restrict__ keys,
                                 uint32_t *__restrict__ vals, unsigned long long mask)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned long long key = flat_key(g, coords[i * 3 + 0], coords[i * 3 + 1], coords[i * 3 + 2]);
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe)
    {
        const unsigned long long prev = atomicCAS(&keys[h], kEmptyKey, key);
        if (prev == kEmptyKey)
        {
            vals[h] = (uint32_t)i;
            return;
        }
        if (prev == key)
        {
            // duplicate coordinate: the lowest row wins (deterministic)
            atomicMin(&vals[h], (uint32_t)i);
            return;
        }
        h = (h + 1) & mask;
    }
}

__device__ __forceinline__ uint32_t mesh_hash_find(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ vals,
                                                   unsigned long long mask, unsigned long long key)
{
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long probe = 0; probe <= mask; ++probe)
    {
        const unsigned long long k = keys[h];
        if (k == key)
            return vals[h];
        if (k == kEmptyKey)
            return kNoVoxel;
        h = (h + 1) & mask;
    }
    return kNoVoxel;
}

// Voxels around the edge of voxel (x,y,z) along each axis, in quad order
// (flexible_dual_grid.py:369-376).
__constant__ int kEdgeNbr[3][4][3] = {
    {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}},
    {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}},
    {{0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}},
};

// One thread per (voxel, axis): the candidate quad (four voxel rows) and whether it is complete.
__global__ void mesh_quads(const int32_t *__restrict__ coords, const uint8_t *__restrict__ flags, long long n, MeshGrid g,
                           const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ vals, unsigned long long mask,
                           uint4 *__restrict__ cand, uint32_t *__restrict__ valid)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * n)
        return;
    const long long i = e / 3;
    const int a = (int)(e - 3 * i);
    uint32_t q[4] = {kNoVoxel, kNoVoxel, kNoVoxel, kNoVoxel};
    bool ok = flags[e] != 0;
    if (ok)
    {
        const long long x = coords[i * 3 + 0], y = coords[i * 3 + 1], z = coords[i * 3 + 2];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            const long long nx = x + kEdgeNbr[a][k][0], ny = y + kEdgeNbr[a][k][1], nz = z + kEdgeNbr[a][k][2];
            const bool inside = nx >= 0 && nx < g.gx && ny >= 0 && ny < g.gy && nz >= 0 && nz < g.gz;
            q[k] = inside ? mesh_hash_find(keys, vals, mask, flat_key(g, nx, ny, nz)) : kNoVoxel;
            ok = ok && q[k] != kNoVoxel;
        }
    }
    cand[e] = make_uint4(q[0], q[1], q[2], q[3]);
    valid[e] = ok ? 1u : 0u;
}

// Mesh vertex of each voxel: (coords + dual) * voxel_size + aabb_min, each
// operation rounded on its own as the reference's separate tensor operations are.
__global__ void mesh_vertices(const int32_t *__restrict__ coords, const float *__restrict__ dual, long long n, MeshGrid g,
                              float *__restrict__ out)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n)
        return;
    const int a = (int)(k % 3);
    out[k] = __fadd_rn(__fmul_rn(__fadd_rn((float)coords[k], dual[k]), g.vs[a]), g.amin[a]);
}

__device__ __forceinline__ void load3(const float *v, uint32_t i, float p[3])
{
    p[0] = v[(size_t)i * 3 + 0];
    p[1] = v[(size_t)i * 3 + 1];
    p[2] = v[(size_t)i * 3 + 2];
}

// cross(b - a, c - a), component by component
__device__ __forceinline__ void tri_cross(const float a[3], const float b[3], const float c[3], float n[3])
{
    const float u0 = __fsub_rn(b[0], a[0]), u1 = __fsub_rn(b[1], a[1]), u2 = __fsub_rn(b[2], a[2]);
    const float w0 = __fsub_rn(c[0], a[0]), w1 = __fsub_rn(c[1], a[1]), w2 = __fsub_rn(c[2], a[2]);
    n[0] = __fsub_rn(__fmul_rn(u1, w2), __fmul_rn(u2, w1));
    n[1] = __fsub_rn(__fmul_rn(u2, w0), __fmul_rn(u0, w2));
    n[2] = __fsub_rn(__fmul_rn(u0, w1), __fmul_rn(u1, w0));
}

// |cross(p1-p0, p2-p0) . cross(p2-p1, p3-p1)| for four entries p0..p3 of a split's index list
__device__ __forceinline__ float split_alignment(const float *v, uint32_t i0, uint32_t i1, uint32_t i2, uint32_t i3)
{
    float p0[3], p1[3], p2[3], p3[3], n0[3], n1[3];
    load3(v, i0, p0);
    load3(v, i1, p1);
    load3(v, i2, p2);
    load3(v, i3, p3);
    tri_cross(p0, p1, p2, n0);
    tri_cross(p1, p2, p3, n1);
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(n0[0], n1[0]), __fmul_rn(n0[1], n1[1])), __fmul_rn(n0[2], n1[2]));
    return fabsf(d);
}

// One thread per complete quad: its triangles (and, in training mode, its middle vertex).
__global__ void mesh_triangles(const uint4 *__restrict__ cand, const uint32_t *__restrict__ valid, const unsigned long long *__restrict__ qoff,
                               long long ne, const float *verts, const float *__restrict__ split_weight, int train,
                               long long nvox, float *vout, int32_t *__restrict__ tris)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne || !valid[e])
        return;
    const long long l = (long long)qoff[e];
    const uint4 q4 = cand[e];
    const uint32_t q[4] = {q4.x, q4.y, q4.z, q4.w};
    if (!train)
    {
        bool first;
        if (split_weight)
        {
            const float w02 = __fmul_rn(split_weight[q[0]], split_weight[q[2]]);
            const float w13 = __fmul_rn(split_weight[q[1]], split_weight[q[3]]);
            first = w02 > w13;
        }
        else
        {
            // The reference forms, for each split's index list t = (t0..t5)
            // (split 1: q0 q1 q2 q0 q2 q3, split 2: q0 q1 q3 q3 q1 q2), the
            // normals cross(t1-t0, t2-t0) and cross(t2-t1, t3-t1) and keeps
            // split 1 when the first alignment is larger (flexible_dual_grid.py:
            // 438-452); the same four entries are used here.  For split 2,
            // t2 == t3, so its alignment is 0.
            const float a0 = split_alignment(verts, q[0], q[1], q[2], q[0]);
            const float a1 = split_alignment(verts, q[0], q[1], q[3], q[3]);
            first = a0 > a1;
        }
        int32_t *t = tris + l * 6;
        if (first)
        {
            t[0] = (int32_t)q[0]; t[1] = (int32_t)q[1]; t[2] = (int32_t)q[2];
            t[3] = (int32_t)q[0]; t[4] = (int32_t)q[2]; t[5] = (int32_t)q[3];
        }
        else
        {
            t[0] = (int32_t)q[0]; t[1] = (int32_t)q[1]; t[2] = (int32_t)q[3];
            t[3] = (int32_t)q[3]; t[4] = (int32_t)q[1]; t[5] = (int32_t)q[2];
        }
        return;
    }
    // training mode (flexible_dual_grid.py:463-474): weighted middle vertex, four triangles
    const float w02 = __fmul_rn(split_weight[q[0]], split_weight[q[2]]);
    const float w13 = __fmul_rn(split_weight[q[1]], split_weight[q[3]]);
    float p0[3], p1[3], p2[3], p3[3];
    load3(verts, q[0], p0);
    load3(verts, q[1], p1);
    load3(verts, q[2], p2);
    load3(verts, q[3], p3);
    const uint32_t mid = (uint32_t)(nvox + l);
#pragma unroll
    for (int c = 0; c < 3; ++c)
    {
        const float m02 = __fdiv_rn(__fadd_rn(p0[c], p2[c]), 2.0f);
        const float m13 = __fdiv_rn(__fadd_rn(p1[c], p3[c]), 2.0f);
        vout[(size_t)mid * 3 + c] = __fdiv_rn(__fadd_rn(__fmul_rn(w02, m02), __fmul_rn(w13, m13)), __fadd_rn(w02, w13));
    }
    int32_t *t = tris + l * 12;
    const uint32_t order[12] = {0, 1, 4, 1, 2, 4, 2, 3, 4, 3, 0, 4};
#pragma unroll
    for (int k = 0; k < 12; ++k)
        t[k] = (int32_t)(order[k] == 4 ? mid : q[order[k]]);
}

// Makes `device` current for the scope of a C ABI call and gives the calling
// thread its previous device back on return.
struct DeviceScope
{
    int prev = -1;
    int dev;
    cudaError_t status;
    explicit DeviceScope(int device) : dev(device)
    {
        cudaGetDevice(&prev);
        status = prev == device ? cudaSuccess : cudaSetDevice(device);
    }
    ~DeviceScope()
    {
        if (prev >= 0 && prev != dev)
            cudaSetDevice(prev);
    }
};

struct Buf
{
    void *p = nullptr;
    size_t cap = 0;
};

cudaError_t grow(Buf &b, size_t bytes)
{
    if (bytes == 0)
        bytes = 16;
    if (b.cap >= bytes)
        return cudaSuccess;
    if (b.p)
        cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    const size_t want = bytes + bytes / 4 + 256;
    const cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        return e;
    }
    b.cap = want;
    return cudaSuccess;
}

} // namespace

struct ovx_fdg_mesh_context
{
    int device = 0;
    std::string err;
    Buf keys, vals, cand, valid, qoff, cub_tmp;
    unsigned long long *host = nullptr;
    // state between begin and finish
    int phase = 0;
    const int32_t *coords = nullptr;
    const float *dual = nullptr;
    const float *split_weight = nullptr;
    long long n = 0, quads = 0;
    int train = 0;
    MeshGrid g{};
};

namespace
{

int mfail(ovx_fdg_mesh_context *c, int status, const std::string &what)
{
    c->err = what;
    c->phase = 0;
    return status;
}

#define MESH_CUDA(call)                                                                                        \
    do                                                                                                         \
    {                                                                                                          \
        const cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                                 \
            return mfail(ctx, e_ == cudaErrorMemoryAllocation ? OVX_FDG_OUT_OF_MEMORY : OVX_FDG_CUDA_ERROR,   \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                                  \
    } while (0)

} // namespace

extern "C" {

int ovx_fdg_mesh_context_create(int device, ovx_fdg_mesh_context **out)
{
    if (!out)
        return OVX_FDG_INVALID_ARGUMENT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    {
        cudaGetLastError();
        return OVX_FDG_INVALID_ARGUMENT;
    }
    ovx_fdg_mesh_context *ctx = new ovx_fdg_mesh_context();
    ctx->device = device;
    if (cudaMallocHost(&ctx->host, 64) != cudaSuccess)
    {
        cudaGetLastError();
        delete ctx;
        return OVX_FDG_OUT_OF_MEMORY;
    }
    *out = ctx;
    return OVX_FDG_OK;
}

void ovx_fdg_mesh_context_destroy(ovx_fdg_mesh_context *ctx)
{
    if (!ctx)
        return;
    const DeviceScope scope(ctx->device);
    for (Buf *b : {&ctx->keys, &ctx->vals, &ctx->cand, &ctx->valid, &ctx->qoff, &ctx->cub_tmp})
        if (b->p)
            cudaFree(b->p);
    if (ctx->host)
        cudaFreeHost(ctx->host);
    delete ctx;
}

const char *ovx_fdg_mesh_last_error(const ovx_fdg_mesh_context *ctx)
{
    return ctx ? ctx->err.c_str() : "";
}

int ovx_fdg_to_mesh_begin(ovx_fdg_mesh_context *ctx, void *stream, const int32_t *coords, const float *dual_vertices,
                          const uint8_t *intersected, const float *split_weight, int64_t num_voxels, const int32_t grid_size[3],
                          const float voxel_size[3], const float aabb_min[3], int32_t train, int64_t *num_vertices,
                          int64_t *num_triangles)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    ctx->phase = 0;
    ctx->err.clear();
    if (!num_vertices || !num_triangles || !grid_size || !voxel_size || !aabb_min || num_voxels < 0)
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "bad argument");
    if (num_voxels > 0 && (!coords || !dual_vertices || !intersected))
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL input");
    if (train && !split_weight)
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "split_weight must be provided in training mode");
    if (num_voxels >= (1ll << 31))
        return mfail(ctx, OVX_FDG_CAPACITY, "more than 2^31-1 voxels");
    MeshGrid g{};
    g.gx = grid_size[0];
    g.gy = grid_size[1];
    g.gz = grid_size[2];
    if (g.gx < 1 || g.gy < 1 || g.gz < 1 || g.gx > (1 << 21) || g.gy > (1 << 21) || g.gz > (1 << 21))
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "grid_size out of range");
    for (int a = 0; a < 3; ++a)
    {
        g.vs[a] = voxel_size[a];
        g.amin[a] = aabb_min[a];
    }
    *num_vertices = 0;
    *num_triangles = 0;
    cudaStream_t st = (cudaStream_t)stream;
    const DeviceScope scope(ctx->device);
    MESH_CUDA(scope.status);
    const long long n = num_voxels, ne = 3 * n;
    unsigned long long cap = 2;
    while (cap < 2ull * (unsigned long long)(n > 0 ? n : 1))
        cap <<= 1;
    MESH_CUDA(grow(ctx->keys, cap * 8));
    MESH_CUDA(grow(ctx->vals, cap * 4));
    MESH_CUDA(grow(ctx->cand, (size_t)(ne + 1) * 16));
    MESH_CUDA(grow(ctx->valid, (size_t)(ne + 1) * 4));
    MESH_CUDA(grow(ctx->qoff, (size_t)(ne + 1) * 8));
    unsigned long long *keys = (unsigned long long *)ctx->keys.p;
    uint32_t *vals = (uint32_t *)ctx->vals.p;
    MESH_CUDA(cudaMemsetAsync(keys, 0xff, cap * 8, st));
    MESH_CUDA(cudaMemsetAsync((uint32_t *)ctx->valid.p + ne, 0, 4, st));
    if (n > 0)
    {
        mesh_hash_insert<<<blocks_for(n, kThreads), kThreads, 0, st>>>(coords, n, g, keys, vals, cap - 1);
        mesh_quads<<<blocks_for(ne, kThreads), kThreads, 0, st>>>(coords, intersected, n, g, keys, vals, cap - 1,
                                                                  (uint4 *)ctx->cand.p, (uint32_t *)ctx->valid.p);
        MESH_CUDA(cudaGetLastError());
    }
    size_t bytes = 0;
    const uint32_t *vin = (const uint32_t *)ctx->valid.p;
    unsigned long long *qoff = (unsigned long long *)ctx->qoff.p;
    MESH_CUDA(cub::DeviceScan::ExclusiveScan(nullptr, bytes, vin, qoff, cub::Sum(), 0ull, (int)(ne + 1), st));
    MESH_CUDA(grow(ctx->cub_tmp, bytes));
    MESH_CUDA(cub::DeviceScan::ExclusiveScan(ctx->cub_tmp.p, bytes, vin, qoff, cub::Sum(), 0ull, (int)(ne + 1), st));
    MESH_CUDA(cudaMemcpyAsync(ctx->host, qoff + ne, 8, cudaMemcpyDeviceToHost, st));
    MESH_CUDA(cudaStreamSynchronize(st));
    const long long L = (long long)ctx->host[0];
    ctx->coords = coords;
    ctx->dual = dual_vertices;
    ctx->split_weight = split_weight;
    ctx->n = n;
    ctx->quads = L;
    ctx->train = train ? 1 : 0;
    ctx->g = g;
    *num_vertices = train ? n + L : n;
    *num_triangles = train ? 4 * L : 2 * L;
    ctx->phase = 1;
    return OVX_FDG_OK;
}

int ovx_fdg_to_mesh_finish(ovx_fdg_mesh_context *ctx, void *stream, float *vertices, int32_t *triangles)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (ctx->phase != 1)
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "ovx_fdg_to_mesh_finish without a successful ovx_fdg_to_mesh_begin");
    ctx->phase = 0;
    const long long n = ctx->n, ne = 3 * n, L = ctx->quads;
    if (n == 0)
        return OVX_FDG_OK;
    if (!vertices || (L > 0 && !triangles))
        return mfail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL output buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const DeviceScope scope(ctx->device);
    MESH_CUDA(scope.status);
    mesh_vertices<<<blocks_for(3 * n, kThreads), kThreads, 0, st>>>(ctx->coords, ctx->dual, n, ctx->g, vertices);
    if (L > 0)
        mesh_triangles<<<blocks_for(ne, kThreads), kThreads, 0, st>>>((const uint4 *)ctx->cand.p, (const uint32_t *)ctx->valid.p,
                                                                     (const unsigned long long *)ctx->qoff.p, ne, vertices,
                                                                     ctx->split_weight, ctx->train, n, vertices, triangles);
    MESH_CUDA(cudaGetLastError());
    return OVX_FDG_OK;
}

} // extern "C"
