/*
 * ovx_fdg.h -- C ABI of the B200 mesh -> flexible dual grid library
 * (libovx_fdg.so).  Plain pointers and sizes; device pointers are CUDA device
 * memory on the context's device; `stream` is a cudaStream_t passed as void*
 * (NULL = legacy default stream).  Calls that take a context make its device
 * current while they run and give the calling thread its previous current
 * device back on return.
 *
 * The entry points replace the reference's CUDA operator for this path:
 *
 *   o_voxel._C.mesh_to_flexible_dual_grid_cuda(vertices, faces, voxel_size,
 *       grid_range, face_weight, boundary_weight, regularization_weight)
 *       -> (voxels int32[N,3], dual_vertices float32[N,3], intersected bool[N,3])
 *     declared in src/convert/api.h:164-172, bound in src/ext.cpp:19,
 *     implemented in src/convert/mesh_to_flexible_dual_grid_gpu/mesh_to_flexible_dual_grid.cu:797-895
 *   -> ovx_fdg_begin + ovx_fdg_finish
 *
 *   o_voxel._C.intersect_occ_cuda(triangles, voxel_size, grid_range) -> int32[N,3]
 *     declared in src/convert/api.h:63-66, bound in src/ext.cpp:21,
 *     implemented in src/convert/mesh_to_flexible_dual_grid_gpu/intersect_qef.cu:896-920
 *   -> ovx_fdg_occupancy_begin + ovx_fdg_occupancy_finish
 *
 * Semantics follow the reference CPU path (src/convert/flexible_dual_grid.cpp):
 * occupancy, intersected flags and dual vertices are bit-identical to it for
 * the floating-point evaluation order documented in the library.  Output rows
 * are in a deterministic order: 8x8x8 bricks in x-fastest order, voxels inside
 * a brick in x-fastest order (the reference GPU order is arbitrary; the
 * reference CPU order is first-touch order).
 *
 * Two calls per conversion: `begin` runs the occupancy stage and returns the
 * number of voxel rows N (one stream synchronisation); the caller then
 * provides output buffers with N rows and `finish` enqueues the quadric and
 * solve stages on the stream and returns without synchronising.  A
 * context holds its device workspace and the state between the two calls; it
 * is not safe to use one context from two threads at once.  Conversions on
 * one context may use different streams: each begin first waits for the work
 * the previous conversion queued, so the workspace is never shared while in use.
 */
#ifndef OVX_FDG_H
#define OVX_FDG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum ovx_fdg_status
{
    OVX_FDG_OK = 0,
    OVX_FDG_INVALID_ARGUMENT = 1, /* bad pointer, size, grid or call order (reference: TORCH_CHECK -> RuntimeError) */
    OVX_FDG_BAD_FACE_INDEX = 2,   /* a face index outside [0, num_vertices) */
    OVX_FDG_CUDA_ERROR = 3,       /* a CUDA runtime call or launch failed */
    OVX_FDG_OUT_OF_MEMORY = 4,    /* workspace allocation failed */
    OVX_FDG_CAPACITY = 5,         /* input or result beyond the indexing limits (2^28-1 faces, 2^31-2 vertices, 2^31-1 voxels) */
    OVX_FDG_INTERNAL = 6          /* a device-side bound (walk length) was hit; results not produced */
};

/* Voxel grid: voxel i along axis a spans [i*voxel_size[a], (i+1)*voxel_size[a])
 * in grid-local coordinates, for grid_min[a] <= i < grid_max[a]
 * (reference grid_range = {grid_min..., grid_max...}, flexible_dual_grid.py:178). */
typedef struct ovx_fdg_grid
{
    float voxel_size[3];
    int32_t grid_min[3];
    int32_t grid_max[3];
} ovx_fdg_grid;

typedef struct ovx_fdg_context ovx_fdg_context;

/* Create a context bound to a CUDA device.  No device memory is allocated until the first call. */
int ovx_fdg_context_create(int device, ovx_fdg_context **out);
void ovx_fdg_context_destroy(ovx_fdg_context *ctx);
/* Human-readable text for a status code, and the last error recorded on a context. */
const char *ovx_fdg_status_string(int status);
const char *ovx_fdg_last_error(const ovx_fdg_context *ctx);
/* Bytes of device workspace the context currently holds. */
int64_t ovx_fdg_workspace_bytes(const ovx_fdg_context *ctx);

/*
 * Instrumentation (no counterpart in the reference, which has no CUDA-side
 * timers).  With profiling on, the context records CUDA events between the
 * pipeline stages of each conversion; ovx_fdg_stage_times waits for the last
 * conversion and writes up to `capacity` stage durations in milliseconds
 * (names from ovx_fdg_stage_name), returning how many it wrote.
 * ovx_fdg_kernel_launches counts the kernels the library itself launched
 * (library scans it calls are not counted).
 */
int ovx_fdg_set_profiling(ovx_fdg_context *ctx, int enable);
int ovx_fdg_stage_times(ovx_fdg_context *ctx, float *ms, int capacity);
const char *ovx_fdg_stage_name(int stage);
int64_t ovx_fdg_kernel_launches(const ovx_fdg_context *ctx);
/*
 * Output row order of the following conversions (full and occupancy-only):
 * OVX_FDG_ORDER_BRICK (default) -- 8x8x8 bricks in x-fastest order, voxels in
 * x-fastest order inside a brick; OVX_FDG_ORDER_Z -- ascending z-order code
 * (ovx_z_order_encode of the voxel coordinates), i.e. the order the
 * reference's examples produce by sorting on o_voxel.serialize.encode_seq
 * (examples/mesh2ovox.py:31-35).  Z-order needs grid_min >= 0 and a multiple
 * of 8 on every axis.  No counterpart in the reference operator.
 */
enum ovx_fdg_order
{
    OVX_FDG_ORDER_BRICK = 0,
    OVX_FDG_ORDER_Z = 1
};
int ovx_fdg_set_output_order(ovx_fdg_context *ctx, int order);

/*
 * Arithmetic of the following full conversions (no counterpart in the
 * reference, whose CPU path sums and solves in FP32 and whose GPU path sums
 * with FP32 atomics).
 * OVX_FDG_PRECISION_EXACT (default): bit-identical to the reference CPU path.
 * OVX_FDG_PRECISION_COMPENSATED: each voxel's quadric, mass point and count
 * are summed in FP32 with two-sum error terms (in the same order) and merged
 * in FP64; regularisation in FP64; the FP32 solve of the rounded quadric is
 * kept unless its error estimate -- the pivoted QR's condition estimate
 * |R00|/|R22| x FLT_EPSILON x the voxel's distance from the grid origin in
 * voxel edges -- exceeds route_tolerance voxel edges, in which case the voxel
 * is solved (and box-constrained) in FP64.  Occupancy and flags are the same
 * in both modes; dual vertices move toward the FP64 result.
 */
enum ovx_fdg_precision
{
    OVX_FDG_PRECISION_EXACT = 0,
    OVX_FDG_PRECISION_COMPENSATED = 1
};
int ovx_fdg_set_precision(ovx_fdg_context *ctx, int precision, float route_tolerance);

/*
 * Work shapes of a context's following conversions (no counterpart in the
 * reference, whose shapes are constants: 16x16 scan tiles,
 * intersect_qef.cu:27-28, and 8^3 bricks, types.cuh:50).  Results do not
 * depend on them; speed does, with the mesh and grid.  NULL restores the
 * defaults (64, 256, 8, 32, 64).  o_voxel picks them per grid size from a
 * table written by the project's tuner (fdg_tune.py).
 *   unit_cells          cells (rows x columns) per unit of work of a large
 *                       (triangle, projection axis) pair, 8..4096
 *   warp_scan_cells     pairs with more cells than this are cut into units, 1..2^20
 *   inline_face_bricks  triangles whose face box spans more 8^3 bricks go to
 *                       the large-triangle face pass, 1..4096
 *   dense_candidates    (triangle, brick) items with more candidate voxels are
 *                       tested by a whole warp, the others through a shared list, 0..512
 *   long_walk           boundary edges whose walk may take more steps are
 *                       walked by a whole warp, 1..2^20
 */
typedef struct ovx_fdg_tuning
{
    int32_t unit_cells;
    int32_t warp_scan_cells;
    int32_t inline_face_bricks;
    int32_t dense_candidates;
    int32_t long_walk;
} ovx_fdg_tuning;
int ovx_fdg_set_tuning(ovx_fdg_context *ctx, const ovx_fdg_tuning *tuning);
int ovx_fdg_get_tuning(const ovx_fdg_context *ctx, ovx_fdg_tuning *tuning);

/*
 * z-order (Morton) codes, o_voxel.serialize.encode_seq / decode_seq with
 * mode='z_order' (serialize.py:7-36, src/serialize/z_order.cu:33-97,
 * src/ext.cpp:28-29): code = interleave of the low 10 bits of x, y, z with x
 * the most significant of each triple; device int32 arrays of length n,
 * enqueued on `stream`.  Coordinates must lie in [0, 1024).
 */
int ovx_z_order_encode(void *stream, const int32_t *x, const int32_t *y, const int32_t *z, int64_t n, int32_t *codes);
int ovx_z_order_decode(void *stream, const int32_t *codes, int64_t n, int32_t *x, int32_t *y, int32_t *z);

/*
 * Hilbert codes, o_voxel.serialize.encode_seq / decode_seq with mode='hilbert'
 * (serialize.py:7-66, src/serialize/hilbert.cu:33-130 (CPU) and :132-240
 * (CUDA), src/ext.cpp:30-31): J. Skilling's transposed Hilbert index of the
 * low 10 bits of x, y, z, its three words interleaved like the z-order code;
 * device int32 arrays of length n, enqueued on `stream`.  Coordinates must lie
 * in [0, 1024).
 */
int ovx_hilbert_encode(void *stream, const int32_t *x, const int32_t *y, const int32_t *z, int64_t n, int32_t *codes);
int ovx_hilbert_decode(void *stream, const int32_t *codes, int64_t n, int32_t *x, int32_t *y, int32_t *z);

/*
 * .vxz attribute packing of a conversion's outputs, as the reference's example
 * does before writing (examples/mesh2ovox.py:51-54): dual_u8[i][a] =
 * uint8(clamp(dual[i][a] * resolution[a] - voxel[i][a], 0, 1) * 255) (float32,
 * truncating), intersected_u8[i] = x + 2y + 4z of the three flags.  Device
 * arrays of n rows, enqueued on `stream`.
 */
int ovx_fdg_pack(void *stream, const int32_t *voxel_indices, const float *dual_vertices, const uint8_t *intersected,
                 int64_t n, const float resolution[3], uint8_t *dual_u8, uint8_t *intersected_u8);

/* Sizes of the last conversion, known after ovx_fdg_begin: out[0] voxel rows,
 * out[1] occupied 8^3 bricks, out[2] quadric records bucketed by brick,
 * out[3] boundary edges, out[4] bricks of the grid; and, after
 * ovx_fdg_sync_status, out[5] voxels the compensated precision mode solved
 * in FP64.  Writes min(capacity, 6) values and returns how many it wrote
 * (negative status on error). */
int ovx_fdg_last_counts(const ovx_fdg_context *ctx, int64_t *out, int capacity);

/*
 * Occupancy stage of mesh -> flexible dual grid.
 *   vertices: device float32 [num_vertices, 3], NOT shifted; origin (host
 *             float[3], may be NULL for zero) is subtracted in float32 exactly
 *             as the reference wrapper does (`vertices - aabb[0]`,
 *             flexible_dual_grid.py:181).
 *   faces:    device int32 or int64 [num_faces, 3] (face_index_bytes = 4 or 8).
 *   grid, weights: as the reference operator (face_weight only gates the face
 *             stage, as in the reference CPU path).
 * On success *num_voxels receives N.  The inputs must stay valid and unchanged until finish returns.
 */
int ovx_fdg_begin(ovx_fdg_context *ctx, void *stream, const float *vertices, int64_t num_vertices,
                  const void *faces, int32_t face_index_bytes, int64_t num_faces, const float *origin,
                  const ovx_fdg_grid *grid, float face_weight, float boundary_weight,
                  float regularization_weight, int64_t *num_voxels);

/*
 * Quadric + solve stages.  Output device buffers with room for N rows:
 *   voxel_indices int32 [N,3], dual_vertices float32 [N,3] (grid-local frame,
 *   like the reference), intersected uint8 [N,3] (0/1, torch.bool layout).
 * Work is enqueued on `stream`; the function returns without synchronising.
 */
int ovx_fdg_finish(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices, float *dual_vertices,
                   uint8_t *intersected);

/*
 * Waits for the work `finish` enqueued on `stream` and reports device-side
 * consistency checks of that stage (the reference has no counterpart: its
 * stages synchronise after every step).  Optional: finish already reports
 * argument and launch errors.
 */
int ovx_fdg_sync_status(ovx_fdg_context *ctx, void *stream);

/*
 * Batched conversion: many meshes, each with its own grid and origin, in one
 * pipeline (no counterpart in the reference, which converts one mesh per
 * call: o_voxel._C.mesh_to_flexible_dual_grid_cuda, src/ext.cpp:19).  All
 * meshes' triangles, bricks and vertices are laid out one mesh after another
 * and every kernel of the conversion runs once over all of them, so a batch
 * costs one host synchronisation (in begin) and one set of launches instead of
 * one per mesh.  Each mesh's result equals what ovx_fdg_begin/ovx_fdg_finish
 * give for it alone, row for row.
 *
 * begin_batch: num_voxels[i] receives mesh i's row count, *total_voxels their
 * sum.  finish_batch: output buffers with room for total_voxels rows; mesh
 * i's rows start at num_voxels[0] + ... + num_voxels[i-1].  Same semantics,
 * order options and errors as the single-mesh calls (an error names the
 * mesh).  Limits over the whole batch: 2^28-1 faces, 2^31-2 vertices, 2^31
 * bricks of the grids.
 */
typedef struct ovx_fdg_mesh
{
    const float *vertices; /* device float32 [num_vertices,3], not shifted */
    int64_t num_vertices;
    const void *faces; /* device int32 or int64 [num_faces,3] */
    int32_t face_index_bytes;
    int64_t num_faces;
    float origin[3]; /* subtracted from the vertices in float32 (aabb[0]) */
    ovx_fdg_grid grid;
} ovx_fdg_mesh;

int ovx_fdg_begin_batch(ovx_fdg_context *ctx, void *stream, const ovx_fdg_mesh *meshes, int32_t num_meshes, float face_weight,
                        float boundary_weight, float regularization_weight, int64_t *num_voxels, int64_t *total_voxels);
int ovx_fdg_finish_batch(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices, float *dual_vertices, uint8_t *intersected);

/*
 * Occupancy only (reference intersect_occ).  triangles: device float32
 * [num_triangles, 3, 3] in grid-local coordinates (already shifted), as the
 * reference operator takes them.  begin returns N; finish writes int32 [N,3].
 */
int ovx_fdg_occupancy_begin(ovx_fdg_context *ctx, void *stream, const float *triangles, int64_t num_triangles,
                            const ovx_fdg_grid *grid, int64_t *num_voxels);
int ovx_fdg_occupancy_finish(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices);

/*
 * Flexible dual grid -> triangle mesh (reference
 * o_voxel.convert.flexible_dual_grid_to_mesh, o_voxel/convert/flexible_dual_grid.py:332-477,
 * with its hashmap src/hash/hash.cu:269-420).  Inputs (device): coords int32
 * [N,3], dual_vertices float32 [N,3] (voxel-relative offsets, as that function
 * takes them), intersected uint8 [N,3], split_weight float32 [N] or NULL;
 * grid_size, voxel_size and aabb_min on the host.  begin finds the quads (one
 * stream synchronisation) and returns the output sizes: num_vertices = N (N +
 * quads in training mode), num_triangles = 2 * quads (4 * quads in training
 * mode, which needs split_weight).  finish writes vertices float32
 * [num_vertices,3] and triangles int32 [num_triangles,3].  A mesh context holds
 * the lookup table and is not safe to use from two threads at once.
 */
typedef struct ovx_fdg_mesh_context ovx_fdg_mesh_context;
int ovx_fdg_mesh_context_create(int device, ovx_fdg_mesh_context **out);
void ovx_fdg_mesh_context_destroy(ovx_fdg_mesh_context *ctx);
const char *ovx_fdg_mesh_last_error(const ovx_fdg_mesh_context *ctx);
int ovx_fdg_to_mesh_begin(ovx_fdg_mesh_context *ctx, void *stream, const int32_t *coords, const float *dual_vertices,
                          const uint8_t *intersected, const float *split_weight, int64_t num_voxels, const int32_t grid_size[3],
                          const float voxel_size[3], const float aabb_min[3], int32_t train, int64_t *num_vertices,
                          int64_t *num_triangles);
int ovx_fdg_to_mesh_finish(ovx_fdg_mesh_context *ctx, void *stream, float *vertices, int32_t *triangles);

/*
 * Occupancy without any allocation (no counterpart in the reference; its
 * operators always allocate).  For hosts that cannot let a library allocate
 * device memory: an application that hands all device memory to its own pool
 * at start-up, or a plugin host whose allocator owns the device, and callers
 * on a latency-critical thread that must not run into the device-wide
 * synchronisation cudaMalloc/cudaFree can imply.  It calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch is one fixed device
 * array inside the library (about 2.2 MiB, held on every device that loads the
 * library until the process exits), sized for grids of at most 32768 8x8x8
 * bricks (for example 256^3).  Larger grids return OVX_FDG_CAPACITY.
 *
 * Same semantics and output row order as ovx_fdg_occupancy_begin/finish:
 * triangles float32 [num_triangles,3,3] in grid-local coordinates on the
 * calling thread's current device; voxel_indices has room for `capacity` rows.
 * *num_voxels receives N; if N > capacity nothing is written and
 * OVX_FDG_CAPACITY is returned.  The call waits once on `stream` (to read N)
 * and returns with the coordinate kernel enqueued on it; because of that wait
 * it cannot run while `stream` is being captured into a CUDA graph, and
 * returns OVX_FDG_INVALID_ARGUMENT without doing anything in that case.  Every
 * call looks up the scratch array's address on the current device (so a
 * cudaDeviceReset between calls is harmless).  All calls on a device share the
 * scratch array, so calls that overlap on the GPU (different streams or
 * threads) race; serialise them.  Each (triangle, axis) pair is scanned by one
 * thread, so a mesh of a few large triangles on a fine grid runs serially
 * inside those threads: the allocating entry points spread such work over
 * whole warps and are the faster choice for low-poly meshes.
 */
int ovx_fdg_occupancy_noalloc(void *stream, const float *triangles, int64_t num_triangles, const ovx_fdg_grid *grid,
                              int32_t *voxel_indices, int64_t capacity, int64_t *num_voxels);

#ifdef __cplusplus
}
#endif

#endif /* OVX_FDG_H */
