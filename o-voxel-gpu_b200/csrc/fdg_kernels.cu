// fdg_kernels.cu -- B200 mesh -> flexible dual grid: kernels, host
// orchestration and the C ABI declared in include/ovx_fdg.h.
//
// Everything is plain SIMT work (scanline rasterisation, bitsets, counting
// sorts, 3x3 solves): nothing is a dense contraction, so no tensor cores.
//
// Data layout in HBM (one conversion):
//   bits    dense occupancy bitmap, brick-major: brick b (x-fastest over the
//           brick grid) owns 16 consecutive 32-bit words; word lz*2+(ly>>2),
//           bit (ly&3)*8+lx (64 B per 8^3 brick, 16.7 MB at grid 512)
//   bbase   exclusive scan of per-brick popcounts = first output row of each
//           brick; rows are brick-major, x-fastest inside a brick
//   roff    exclusive scan of per-brick record counts; records (12 B) are the
//           quadric contributions landing in a brick, bucketed by brick:
//             event    {t, 0<<30 | w<<10 | v<<6 | u<<2 | axis, float z}
//                      one per scanline event and brick it touches; (u,v,w) is
//                      the event's base voxel in projection coordinates,
//                      relative to the brick (u,v offset by one)
//             face     {t, 1<<30 | local voxel, 0}
//             boundary {e, 2<<30 | local voxel, 0}, e = index in the
//                      boundary edge list, which is sorted by (v_min, v_max)
//   qtab    plane quadric per triangle (10 floats in a 12-float row, read as 16-byte loads)
//   contrib per-voxel contribution lists, 8 B entries {order key, payload};
//           each brick reserves its lists' exact room with one atomic (the
//           total is known after begin: 4 per scanline event, 1 per face or
//           boundary record)
//   vlist   per output row: first entry (40 bits) | entry count << 40 | sorted << 63
//   estage, fstage  event and face records staged by the count pass (16 B,
//           {brick, t, code, z} and {brick, t, code, rank in the brick}); both
//           live in one arena that the contribution lists reuse once the
//           staged records are in their buckets
//   clist   voxels left to the constrained search, in the record buffer (dead
//           once the lists are built); when it is full the search runs inline
//   btab    line quadric per boundary edge (10 floats in a 12-float row)
//
// begin (ends with the one host synchronisation of a conversion):
//   tri_events<COUNT>   one (triangle, axis) per lane: scanline events (FP64,
//                       reference arithmetic) set occupancy bits, count event
//                       records per brick and stage them; the quadric table is
//                       written; large pairs are listed
//   large_rows<COUNT>   the listed pairs, cut into units of a few rows
//   compaction          brick popcounts, scans -> N, active bricks
//   edges               undirected edges bucketed by smaller vertex; edges
//                       used once -> boundary list
//   face_records<COUNT> one triangle per lane: face tests, records counted and
//                       staged; triangles over many bricks are listed
//   large_faces<COUNT>  the listed triangles' (triangle, brick) items, one per lane
//   boundary_records<COUNT>, scan -> record offsets
//   (the edges run on a second stream beside the scanline pass)
// finish (no synchronisation):
//   bucket_records      staged event records -> brick buckets, a cursor per brick
//   place_records       staged face records -> their ranks in the buckets
//                       (when a staging buffer overflowed, the generators rerun
//                       in FILL mode and write the records instead)
//   boundary_records<FILL>
//   brick_lists         one CTA per active brick: records -> per-voxel
//                       contribution lists {key, payload} (a counting sort by
//                       voxel), staged and the short ones sorted in shared
//                       memory when the brick's lists fit there
//   voxel_accumulate    one thread per voxel: sorts its list by key unless it is
//                       marked sorted, sums it sequentially in FP32 in that order
//                       (bit-identical to the reference CPU sums), regularises,
//                       CPQR-solves
//   constrained_solve   box-constrained search for the few voxels whose
//                       unconstrained solution leaves the voxel
//
// Contribution order keys (32 bit, unique per voxel; ascending = reference CPU
// order, flexible_dual_grid.cpp:173-283, :298-414, :741-757), F = triangles of
// the conversion (all meshes of a batch; F < 2^28, so every key < 16F < 2^32):
//   intersection  (t*3 + axis)*4 + (1-dy)*2 + (1-dx)     in [0, 12F)
//   face          12F + t                                in [12F, 13F)
//   boundary      13F + e   (edge list index; the list is in (v_min, v_max)
//                           order, and there are at most 3F boundary edges)
#include "ovx_fdg.h"
#include "fdg_device.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <type_traits>

using namespace ovx;

namespace
{

// Work shapes (defaults; a context may be tuned, ovx_fdg_set_tuning):
constexpr int kInlineFaceBricks = 8; // triangles whose face box spans more bricks go to large_faces
constexpr int kUnitCells = 64;        // cells per unit of work of a large (triangle, axis) pair
constexpr int kThreads = 256;
constexpr int kConsumeThreads = 128;
constexpr int kListStage = 1024; // contributions of a brick that brick_lists stages (and sorts) in shared memory
// vlist word: first entry (bits 0-39) | count (bits 40-62) | sorted flag (bit 63)
constexpr uint32_t kListCountMax = (1u << 23) - 1u;
constexpr unsigned long long kListSorted = 1ull << 63;
#ifndef OVX_FDG_WARP_SORT_MIN
#define OVX_FDG_WARP_SORT_MIN 16
#endif
constexpr int kWarpSortMin = OVX_FDG_WARP_SORT_MIN; // lists this long or longer are ordered by the whole warp

// device counter words
enum
{
    C_SCAN_LARGE = 0,
    C_FACE_LARGE = 1,
    C_BOUNDARY = 2,
    C_STATUS = 3,
    C_CONSTRAINED = 4,
    C_FSTAGED = 5,
    C_LONG = 6,
    C_HUGE = 7,
    C_LUNITS = 8,  // units of work of the large (triangle, axis) pairs
    C_FUNITS = 9,  // units of work of the large triangles' face boxes
    C_BLONG = 10,  // boundary edges walked by a whole warp
    C_ROUTED = 11, // compensated precision: voxels solved in FP64
    C_CONTRIB = 12, // 64-bit word (12, 13): contribution entries reserved by brick_lists
    C_ESTAGED = 14, // 64-bit pair (14, 15), added to as one word: scanline event records staged,
    C_EVENTS = 15,  // and scanline events (each yields four contributions)
    C_WORDS = 16
};
static_assert(C_CONTRIB % 2 == 0 && C_ESTAGED % 2 == 0 && C_EVENTS == C_ESTAGED + 1, "64-bit counters are 8-byte aligned words");
enum
{
    ST_BAD_INDEX = 1,
    ST_WALK_GUARD = 2,
    ST_LIST_OVERFLOW = 4,
    ST_REPLAY = 8
};

enum Mode
{
    COUNT = 0,
    FILL = 1
};

constexpr uint32_t kRecFace = 1u << 30;
constexpr uint32_t kRecBoundary = 2u << 30;
constexpr long long kMaxTriangles = (1ll << 28) - 1; // 32-bit order keys: 16F < 2^32

struct Rec
{
    uint32_t a, b, c;
};

// (u, v, w) are coordinates along (ax0, ax1, ax2) of projection axis ax2.
__device__ __forceinline__ void place(int ax2, int u, int v, int w, int &x, int &y, int &z)
{
    x = ax2 == 0 ? w : (ax2 == 1 ? v : u);
    y = ax2 == 0 ? u : (ax2 == 1 ? w : v);
    z = ax2 == 0 ? v : (ax2 == 1 ? u : w);
}

// One mesh of a conversion.  A batched conversion lays its meshes' triangles,
// bricks and vertices out one mesh after another in global index spaces; a
// mesh's entries there start at tri0, brick0 and vert0 (all 0 for a single
// mesh), and its output rows at row0.
struct Mesh
{
    Grid g;
    const float *verts;
    long long nv;
    const void *faces; // NULL: triangle soup, vertex 3t+k
    long long nf;
    float ox, oy, oz;
    int fbytes; // bytes per face index (4 or 8)
    long long tri0, brick0, vert0, row0;
};

template <typename IdxT>
__device__ __forceinline__ bool tri_load(const Mesh &M, long long t, float v[3][3])
{
    long long idx[3];
    const float o[3] = {M.ox, M.oy, M.oz};
    return load_triangle<IdxT>(M.verts, M.nv, (const IdxT *)M.faces, t, o, v, idx);
}

// Triangle t (local to its mesh): single conversions know the face index type
// at compile time; batched ones read it from the mesh.
template <bool B, typename IdxT>
__device__ __forceinline__ bool tri_load_m(const Mesh &M, long long t, float v[3][3])
{
    if constexpr (B)
        return M.fbytes == 8 ? tri_load<long long>(M, t, v) : tri_load<int>(M, t, v);
    else
        return tri_load<IdxT>(M, t, v);
}

// Mesh of a global index: the last of the n meshes whose first index
// first(i) is at most x (first is non-decreasing).
template <typename First>
__device__ __forceinline__ int seg_find(int n, long long x, First first)
{
    int lo = 0, hi = n;
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if (first(mid) <= x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// The mesh of a conversion: the single mesh in the kernel's parameters, or
// mesh s of a batch's table in global memory.
template <bool B, typename Args>
__device__ __forceinline__ const Mesh &mesh_of(const Args &A, int s)
{
    if constexpr (B)
        return A.segs[s];
    else
        return A.m;
}

template <bool B, typename Args>
__device__ __forceinline__ int seg_of_tri(const Args &A, long long t)
{
    if constexpr (B)
        return seg_find(A.nseg, t, [&](int i) { return A.segs[i].tri0; });
    else
        return 0;
}

template <bool B, typename Args>
__device__ __forceinline__ int seg_of_brick(const Args &A, long long b)
{
    if constexpr (B)
        return seg_find(A.nseg, b, [&](int i) { return A.segs[i].brick0; });
    else
        return 0;
}

template <bool B, typename Args>
__device__ __forceinline__ int seg_of_vert(const Args &A, long long v)
{
    if constexpr (B)
        return seg_find(A.nseg, v, [&](int i) { return A.segs[i].vert0; });
    else
        return 0;
}

template <bool B, typename Args>
__device__ __forceinline__ int seg_of_row(const Args &A, long long r)
{
    if constexpr (B)
        return seg_find(A.nseg, r, [&](int i) { return A.segs[i].row0; });
    else
        return 0;
}

__device__ __forceinline__ void vertex_load(const Mesh &M, long long i, float p[3])
{
    p[0] = M.verts[i * 3 + 0] - M.ox;
    p[1] = M.verts[i * 3 + 1] - M.oy;
    p[2] = M.verts[i * 3 + 2] - M.oz;
}

// z-order (Morton) codes with x as the most significant coordinate of each bit
// triple, as o_voxel.serialize.encode_seq builds them (serialize/z_order.cu:33-97).
__host__ __device__ __forceinline__ uint32_t spread3_10(uint32_t v)
{
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 10; ++i)
        r |= ((v >> i) & 1u) << (3 * i);
    return r;
}

__host__ __device__ __forceinline__ uint32_t compact3_10(uint32_t c)
{
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 10; ++i)
        r |= ((c >> (3 * i)) & 1u) << i;
    return r;
}

// Local index lx + 8ly + 64lz of an 8^3 brick -> its 9-bit z-order rank.
__device__ __forceinline__ int local_morton(int lv)
{
    const uint32_t lx = (uint32_t)lv & 7u, ly = ((uint32_t)lv >> 3) & 7u, lz = (uint32_t)lv >> 6;
    return (int)((spread3_10(lx) << 2) | (spread3_10(ly) << 1) | spread3_10(lz));
}

__device__ __forceinline__ unsigned long long brick_morton(unsigned long long bx, unsigned long long by, unsigned long long bz)
{
    unsigned long long r = 0;
#pragma unroll
    for (int i = 0; i < 21; ++i)
        r |= (((bx >> i) & 1ull) << (3 * i + 2)) | (((by >> i) & 1ull) << (3 * i + 1)) | (((bz >> i) & 1ull) << (3 * i));
    return r;
}

__device__ __forceinline__ void brick_origin(const Grid &g, long long b, int o[3])
{
    o[0] = g.gmin[0] + (int)(b % g.nb[0]) * kBrick;
    o[1] = g.gmin[1] + (int)((b / g.nb[0]) % g.nb[1]) * kBrick;
    o[2] = g.gmin[2] + (int)(b / ((long long)g.nb[0] * g.nb[1])) * kBrick;
}

// ===========================================================================
// record generation
// ===========================================================================
// Work shapes of the record generators (ovx_fdg_tuning).
struct Tuning
{
    int unit_cells, scan_work, inline_face_bricks, dense_candidates, long_walk;
};

struct GenArgs
{
    Tuning tune;
    Mesh m;
    const Mesh *segs; // batched conversions: the meshes (global memory)
    int nseg;
    uint32_t *bits;
    uint32_t *rcnt;                 // records per brick (COUNT) / cursor (FILL)
    const unsigned long long *roff; // FILL
    Rec *rec;                       // FILL
    float *qtab;                    // COUNT of the intersection pass
    float *btab;                    // FILL of the boundary pass
    uint4 *fstage;                  // COUNT of the face pass: face records {brick, t, code, 0} (NULL: off)
    uint32_t fstage_cap;
    uint4 *estage;                  // COUNT of the scanline pass: event records {brick, t, code, z} (NULL: off)
    uint32_t estage_cap;
    uint32_t *counters;
    uint32_t *scan_large;
    uint32_t *scan_units; // per listed pair: its units of work, then (scanned) its first unit
    uint32_t scan_large_cap;
    uint32_t *face_large;
    uint32_t *face_units; // the same for the listed triangles
    uint32_t face_large_cap;
    const unsigned long long *bkeys;
    uint32_t bkeys_cap;
    uint32_t *blong; // boundary edges with long walks (their index in bkeys)
    uint32_t blong_cap;
};

// Add n to rcnt[b] once per group of lanes of the calling warp that target the
// same brick (neighbouring triangles mostly write the same bricks); returns the
// value of the counter before this lane's share.
__device__ __forceinline__ uint32_t agg_add(uint32_t *cnt, long long b, uint32_t n)
{
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, (unsigned long long)b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    // exclusive prefix of n over the lower lanes of the group
    uint32_t pre = 0, tot = 0;
    for (unsigned m = peers; m; m &= m - 1u)
    {
        const int l = __ffs(m) - 1;
        const uint32_t v = __shfl_sync(peers, n, l);
        if (l < lane)
            pre += v;
        tot += v;
    }
    uint32_t base = 0;
    if (lane == leader)
        base = atomicAdd(&cnt[b], tot);
    base = __shfl_sync(peers, base, leader);
    return base + pre;
}

// One record for brick b (scanline events and boundary walks; these call sites
// sit in divergent loops, where plain atomics beat warp aggregation).
template <int M>
__device__ __forceinline__ void put_record(const GenArgs &A, long long b, uint32_t a0, uint32_t a1, uint32_t a2)
{
    if (M == COUNT)
        atomicAdd(&A.rcnt[b], 1u);
    else
    {
        const uint32_t k = atomicAdd(&A.rcnt[b], 1u);
        const unsigned long long base = A.roff[b];
        if (k >= A.roff[b + 1] - base)
        {
            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_REPLAY);
            return;
        }
        Rec r;
        r.a = a0;
        r.b = a1;
        r.c = a2;
        A.rec[base + k] = r;
    }
}

// Records of one scanline event kept for staging (one brick each, at most four).
struct EventStage
{
    uint32_t n;
    uint32_t b[4], code[4];
    uint32_t zb, t;
};

// Scanline event sink: (COUNT) sets the occupancy bits of the four voxels
// around the grid line and counts one record per distinct brick, optionally
// keeping the records for staging; (FILL) writes those records.
template <int M>
struct EventSink
{
    const GenArgs &A;
    const Mesh &Ms; // the triangle's mesh (its grid, bitmap and first brick)
    uint32_t t;     // global triangle index
    int ax2;
    EventStage *es = nullptr;
    __device__ __forceinline__ void operator()(int xi, int yi, int zi, float, float, double z) const
    {
        const Grid &g = Ms.g;
        uint32_t *const bits = A.bits + Ms.brick0 * kWordsPerBrick;
        long long w[4];
        uint32_t m[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            int x, y, zz;
            place(ax2, xi + (k >> 1), yi + (k & 1), zi, x, y, zz);
            uint32_t bit;
            w[k] = voxel_word(g, x, y, zz, bit);
            m[k] = 1u << bit;
        }
        if (M == COUNT)
        {
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                bool dup = false;
#pragma unroll
                for (int j = 0; j < k; ++j)
                    dup |= (w[j] == w[k]);
                if (dup)
                    continue;
                uint32_t mk = m[k];
#pragma unroll
                for (int j = k + 1; j < 4; ++j)
                    if (w[j] == w[k])
                        mk |= m[j];
                atomicOr(&bits[w[k]], mk);
            }
        }
        const uint32_t zb = __float_as_uint((float)z);
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            const long long b = w[k] >> 4;
            bool dup = false;
#pragma unroll
            for (int j = 0; j < k; ++j)
                dup |= ((w[j] >> 4) == b);
            if (dup)
                continue;
            uint32_t code = 0;
            if (M == FILL || es)
            {
                int o[3];
                brick_origin(g, b, o);
                const int ax0 = (ax2 + 1) % 3, ax1 = (ax2 + 2) % 3;
                const int o0 = ax0 == 0 ? o[0] : (ax0 == 1 ? o[1] : o[2]);
                const int o1 = ax1 == 0 ? o[0] : (ax1 == 1 ? o[1] : o[2]);
                const int o2 = ax2 == 0 ? o[0] : (ax2 == 1 ? o[1] : o[2]);
                code = (uint32_t)ax2 | ((uint32_t)(xi - o0 + 1) << 2) | ((uint32_t)(yi - o1 + 1) << 6) |
                       ((uint32_t)(zi - o2) << 10);
            }
            put_record<M>(A, Ms.brick0 + b, t, code, zb);
            if (M == COUNT && es)
            {
                es->b[es->n] = (uint32_t)(Ms.brick0 + b);
                es->code[es->n] = code;
                ++es->n;
            }
        }
        if (M == COUNT && es)
        {
            es->zb = zb;
            es->t = t;
        }
    }
};

constexpr int kEventThreads = 128;   // scanline pass: one (triangle, axis) per lane
constexpr int kWarpScanWork = 256;   // (triangle, axis) pairs with more row x column work go to large_rows
constexpr int kDenseCandidates = 32; // (triangle, brick) items with more candidates are tested by the whole warp

struct EventWarp
{
    double t[3][3][32]; // sorted vertices (projection coordinates) of each lane's (triangle, axis)
    long long ta[32];   // each lane's pair: 3 * triangle + axis (global triangle index)
    int seg[32];        // each lane's mesh (batched conversions)
    int start[32], mid[32]; // first row of the lane's rows, and the row where the second edge pair starts
    int clo[32], chi[32];   // columns of the lane's rows: [clo, chi)
};

// Largest lane l with v(l) <= x, for v non-decreasing over the lanes (x >= v(0)).
__device__ __forceinline__ int owner_lane(uint32_t v, uint32_t x)
{
    int l = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
    {
        const int c = l + step;
        const uint32_t vc = __shfl_sync(0xffffffffu, v, c & 31);
        if (c < 32 && vc <= x)
            l = c;
    }
    return l;
}

__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t x, uint32_t &total)
{
    const int lane = threadIdx.x & 31;
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d)
            incl += y;
    }
    total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - x;
}

// A large (triangle, axis) pair is cut into units of about `unit` cells:
// blocks of rb rows of narrow pairs, column chunks (nch per row) of wide ones.
struct LargeSplit
{
    int rb, nch;
};

__device__ __forceinline__ LargeSplit large_split(int cols, int unit)
{
    if (cols >= unit)
        return {1, (cols + unit - 1) / unit};
    return {unit / cols, 1};
}

// The rows of the warp's (triangle, axis) pairs (lane l: nrows rows from
// E.start[l]) spread over the lanes 32 at a time, and the column crossings of
// those rows again 32 at a time, so the FP64 event arithmetic runs on full
// warps whatever the pairs' sizes.  COUNT marks the occupancy bits, counts
// event records per brick and stages them; FILL writes the records.
template <int M, bool B>
__device__ __forceinline__ void event_rows(const GenArgs &A, EventWarp &E, const int lane, const uint32_t nrows)
{
    uint32_t nrow_all;
    const uint32_t rstart = warp_exclusive_scan(nrows, nrow_all);
    __syncwarp();
    for (uint32_t rb = 0; rb < nrow_all; rb += 32)
    {
        // this lane's row: owner pair ol, row yi
        const uint32_t r = rb + (uint32_t)lane;
        const int ol = owner_lane(rstart, r);
        const uint32_t ors = __shfl_sync(0xffffffffu, rstart, ol);
        const int oax2 = (int)(E.ta[ol] % 3);
        RowSetup rs;
        rs.t3x = rs.t3z = rs.t4x = rs.t4z = 0.0;
        rs.x0 = rs.x1 = 0;
        int yi = 0;
        if (r < nrow_all)
        {
            AxisScan s;
#pragma unroll
            for (int k = 0; k < 3; ++k)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    s.t[k][c] = E.t[k][c][ol];
            s.start = E.start[ol];
            s.mid = E.mid[ol];
            s.end = 0;
            s.ax2 = oax2;
            s.ax0 = (oax2 + 1) % 3;
            s.ax1 = (oax2 + 2) % 3;
            yi = s.start + (int)(r - ors);
            const Mesh &Mo = mesh_of<B>(A, B ? E.seg[ol] : 0);
            row_setup(s, yi, E.clo[ol], E.chi[ol], Mo.g, rs);
        }
        const uint32_t ncol = rs.x1 > rs.x0 ? (uint32_t)(rs.x1 - rs.x0) : 0u;
        uint32_t ncol_all;
        const uint32_t cstart = warp_exclusive_scan(ncol, ncol_all);
        for (uint32_t cb = 0; cb < ncol_all; cb += 32)
        {
            // this lane's column crossing: owner row lane rl
            const uint32_t c = cb + (uint32_t)lane;
            const int rl = owner_lane(cstart, c);
            RowSetup cr;
            cr.t3x = __shfl_sync(0xffffffffu, rs.t3x, rl);
            cr.t3z = __shfl_sync(0xffffffffu, rs.t3z, rl);
            cr.t4x = __shfl_sync(0xffffffffu, rs.t4x, rl);
            cr.t4z = __shfl_sync(0xffffffffu, rs.t4z, rl);
            cr.x0 = __shfl_sync(0xffffffffu, rs.x0, rl);
            cr.x1 = 0;
            const int cyi = __shfl_sync(0xffffffffu, yi, rl);
            const int col = __shfl_sync(0xffffffffu, ol, rl);
            const uint32_t ccs = __shfl_sync(0xffffffffu, cstart, rl);
            EventStage es;
            es.n = 0;
            if (c < ncol_all)
            {
                const long long cta = E.ta[col];
                const int cax2 = (int)(cta % 3);
                const int xi = cr.x0 + (int)(c - ccs);
                const Mesh &Mc = mesh_of<B>(A, B ? E.seg[col] : 0);
                const Grid &g = Mc.g;
                double z;
                int zi;
                col_event(cr, xi, (cax2 + 1) % 3, cax2, g, z, zi);
                if (zi >= g.gmin[cax2] && zi < g.gmax[cax2])
                {
                    EventSink<M> sink{A, Mc, (uint32_t)(cta / 3), cax2, (M == COUNT && A.estage) ? &es : nullptr};
                    sink(xi, cyi, zi, 0.0f, 0.0f, z);
                }
            }
            if (M == COUNT && A.estage)
            {
                // stage this round's records: one reservation for the warp; the
                // round's events are counted (four contributions each)
                uint32_t tot;
                const uint32_t off = warp_exclusive_scan(es.n, tot);
                const uint32_t nev = (uint32_t)__popc(__ballot_sync(0xffffffffu, es.n > 0u));
                uint32_t base = 0;
                if (lane == 0 && tot)
                    base = (uint32_t)atomicAdd((unsigned long long *)&A.counters[C_ESTAGED],
                                               ((unsigned long long)nev << 32) | (unsigned long long)tot);
                base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if ((uint32_t)k < es.n)
                    {
                        const unsigned long long pos = (unsigned long long)base + off + k;
                        if (pos < A.estage_cap)
                            A.estage[pos] = make_uint4(es.b[k], es.t, es.code[k], es.zb);
                    }
            }
        }
    }
}

// Scanline events (flexible_dual_grid.cpp:195-283), one (triangle, axis) per
// lane.  The rows of the warp's 32 pairs are spread over the lanes 32 at a
// time, and the column crossings of those rows again 32 at a time, so the FP64
// event arithmetic runs on full warps whatever the triangles' sizes.  COUNT
// marks the occupancy bits and counts event records per brick (and writes the
// quadric table); FILL writes the records.
template <int M, typename IdxT, bool B>
__global__ void __launch_bounds__(kEventThreads) tri_events(GenArgs A)
{
    __shared__ EventWarp EW[kEventThreads / 32];
    const int lane = threadIdx.x & 31;
    EventWarp &E = EW[threadIdx.x >> 5];
    const long long ta = (long long)blockIdx.x * blockDim.x + threadIdx.x; // global (triangle, axis)
    uint32_t nrows = 0;
    if (ta < 3 * A.m.nf)
    {
        const long long t = ta / 3;
        const int ax2 = (int)(ta - 3 * t);
        const int sg = seg_of_tri<B>(A, t);
        const Mesh &Ms = mesh_of<B>(A, sg);
        const Grid &g = Ms.g;
        float v[3][3];
        if (!tri_load_m<B, IdxT>(Ms, t - Ms.tri0, v))
        {
            if (M == COUNT)
                atomicOr(&A.counters[C_STATUS], (uint32_t)ST_BAD_INDEX);
        }
        else
        {
            if (M == COUNT && ax2 == 0 && A.qtab)
            {
                float q[10];
                tri_quadric(v, q);
#pragma unroll
                for (int i = 0; i < 10; ++i)
                    A.qtab[t * 12 + i] = q[i];
            }
            AxisScan s;
            axis_setup(v, ax2, g, s);
            const int rows = s.end - s.start;
            if (rows > 0)
            {
                int clo, chi;
                axis_col_bounds(s, g, clo, chi);
                if ((long long)rows * (long long)(chi - clo + 1) > A.tune.scan_work)
                {
                    if (M == COUNT)
                    {
                        const uint32_t slot = atomicAdd(&A.counters[C_SCAN_LARGE], 1u);
                        if (slot < A.scan_large_cap)
                        {
                            const LargeSplit sp = large_split(chi - clo + 1, A.tune.unit_cells);
                            A.scan_large[slot] = (uint32_t)ta;
                            A.scan_units[slot] = (uint32_t)((rows + sp.rb - 1) / sp.rb * sp.nch);
                        }
                        else
                            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
                    }
                }
                else
                {
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            E.t[k][c][lane] = s.t[k][c];
                    E.start[lane] = s.start;
                    E.mid[lane] = s.mid;
                    E.clo[lane] = INT_MIN;
                    E.chi[lane] = INT_MAX;
                    E.ta[lane] = ta;
                    E.seg[lane] = sg;
                    nrows = (uint32_t)rows;
                }
            }
        }
    }
    __syncwarp();
    event_rows<M, B>(A, E, lane, nrows);
}

// In-place exclusive scan of the unit counts of a work list: entry i of
// `units` becomes the first unit of list entry i, entry n the total, which
// also goes to counters[total_word].  n = min(counters[count_word], cap) is
// known only on the device, so the scan covers the capacity in tiles of
// kUnitTile entries (entries from n on count as 0) in three passes: tile
// sums, one CTA scanning the tile sums, then each tile scanning its entries
// from its offset.  A total of 2^32 units or more sets the list-overflow status.
constexpr int kUnitTile = 1024;

__device__ __forceinline__ unsigned long long block_exclusive_u64(unsigned long long v, unsigned long long *wsum,
                                                                  unsigned long long &total)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d)
            incl += y;
    }
    if (lane == 31)
        wsum[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        const int nw = blockDim.x >> 5;
        unsigned long long w = lane < nw ? wsum[lane] : 0ull;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d)
                w += y;
        }
        if (lane < nw)
            wsum[lane] = w;
    }
    __syncthreads();
    total = wsum[(blockDim.x >> 5) - 1];
    const unsigned long long ex = (warp > 0 ? wsum[warp - 1] : 0ull) + incl - v;
    __syncthreads();
    return ex;
}

__global__ void __launch_bounds__(kUnitTile) unit_tile_sums(const uint32_t *__restrict__ units, uint32_t cap,
                                                            const uint32_t *__restrict__ counters, int count_word,
                                                            unsigned long long *__restrict__ tile_sum)
{
    __shared__ unsigned long long wsum[32];
    const uint32_t n = min(counters[count_word], cap);
    const uint32_t i = blockIdx.x * kUnitTile + threadIdx.x;
    unsigned long long total;
    block_exclusive_u64(i < n ? units[i] : 0u, wsum, total);
    if (threadIdx.x == 0)
        tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) unit_tile_offsets(unsigned long long *__restrict__ tile_sum, uint32_t ntiles,
                                                           uint32_t *__restrict__ units, uint32_t cap, uint32_t *__restrict__ counters,
                                                           int count_word, int total_word)
{
    __shared__ unsigned long long wsum[32];
    const int tid = threadIdx.x;
    const uint32_t per = (ntiles + blockDim.x - 1) / blockDim.x;
    const uint32_t b0 = min(ntiles, (uint32_t)tid * per), b1 = min(ntiles, b0 + per);
    unsigned long long sum = 0;
    for (uint32_t i = b0; i < b1; ++i)
        sum += tile_sum[i];
    unsigned long long total;
    unsigned long long run = block_exclusive_u64(sum, wsum, total);
    for (uint32_t i = b0; i < b1; ++i)
    {
        const unsigned long long t = tile_sum[i];
        tile_sum[i] = run;
        run += t;
    }
    if (tid == 0)
    {
        const uint32_t n = min(counters[count_word], cap);
        if (total >= (1ull << 32))
        {
            atomicOr(&counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
            total = 0;
        }
        units[n] = (uint32_t)total;
        counters[total_word] = (uint32_t)total;
    }
}

__global__ void __launch_bounds__(kUnitTile) unit_tile_scan(uint32_t *__restrict__ units, uint32_t cap,
                                                            const uint32_t *__restrict__ counters, int count_word,
                                                            const unsigned long long *__restrict__ tile_sum)
{
    __shared__ unsigned long long wsum[32];
    const uint32_t n = min(counters[count_word], cap);
    const uint32_t i = blockIdx.x * kUnitTile + threadIdx.x;
    const uint32_t u = i < n ? units[i] : 0u;
    unsigned long long total;
    const unsigned long long ex = block_exclusive_u64(u, wsum, total);
    if (i < n)
        units[i] = (uint32_t)(tile_sum[blockIdx.x] + ex);
}

// Entry i of a scanned unit list with units[i] <= u < units[i + 1] (u below units[n]).
__device__ __forceinline__ uint32_t unit_owner(const uint32_t *__restrict__ units, uint32_t n, uint32_t u)
{
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (units[mid] <= u)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Large (triangle, axis) pairs, cut into units of about tune.unit_cells cells (a
// block of rows, or a chunk of one row's columns): one unit per lane, 32 per
// warp, the rows and column crossings of the warp's units spread over the
// lanes as for the other pairs.
template <int M, typename IdxT, bool B>
__global__ void __launch_bounds__(kEventThreads) large_rows(GenArgs A)
{
    __shared__ EventWarp EW[kEventThreads / 32];
    const int lane = threadIdx.x & 31;
    EventWarp &E = EW[threadIdx.x >> 5];
    const uint32_t n = min(A.counters[C_SCAN_LARGE], A.scan_large_cap);
    const uint32_t total = A.counters[C_LUNITS];
    const int wpb = blockDim.x >> 5;
    const long long stride = (long long)gridDim.x * wpb * 32;
    for (long long ub = ((long long)blockIdx.x * wpb + (threadIdx.x >> 5)) * 32; ub < (long long)total; ub += stride)
    {
        const long long u = ub + lane;
        uint32_t nrows = 0;
        if (u < (long long)total)
        {
            const uint32_t i = unit_owner(A.scan_units, n, (uint32_t)u);
            const uint32_t ta = A.scan_large[i];
            const long long t = ta / 3;
            const int ax2 = (int)(ta - 3 * t);
            const int sg = seg_of_tri<B>(A, t);
            const Mesh &Ms = mesh_of<B>(A, sg);
            float v[3][3];
            if (tri_load_m<B, IdxT>(Ms, t - Ms.tri0, v))
            {
                AxisScan s;
                axis_setup(v, ax2, Ms.g, s);
                int clo, chi;
                axis_col_bounds(s, Ms.g, clo, chi);
                const LargeSplit sp = large_split(chi - clo + 1, A.tune.unit_cells);
                const int j = (int)((uint32_t)u - A.scan_units[i]);
                const int ch = j % sp.nch;
                const int r0 = s.start + (j / sp.nch) * sp.rb;
                const int r1 = min(s.end, r0 + sp.rb);
                if (r1 > r0)
                {
#pragma unroll
                    for (int k = 0; k < 3; ++k)
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                            E.t[k][c][lane] = s.t[k][c];
                    E.start[lane] = r0;
                    E.mid[lane] = s.mid;
                    E.clo[lane] = ch == 0 ? INT_MIN : clo + ch * A.tune.unit_cells;
                    E.chi[lane] = ch == sp.nch - 1 ? INT_MAX : clo + (ch + 1) * A.tune.unit_cells;
                    E.ta[lane] = ta;
                    E.seg[lane] = sg;
                    nrows = (uint32_t)(r1 - r0);
                }
            }
        }
        __syncwarp();
        event_rows<M, B>(A, E, lane, nrows);
        __syncwarp();
    }
}

// Face box of a triangle restricted to the brick with origin o, as local
// [lo, hi) per axis; false if empty.
__device__ __forceinline__ bool brick_box(const int bmin[3], const int bmax[3], const int o[3], int lo[3], int hi[3])
{
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        lo[a] = (bmin[a] > o[a] ? bmin[a] : o[a]) - o[a];
        hi[a] = (bmax[a] < o[a] + 8 ? bmax[a] : o[a] + 8) - o[a];
        ok = ok && hi[a] > lo[a];
    }
    return ok;
}

// Word w of a brick's occupancy restricted to the local box [lo, hi).
__device__ __forceinline__ uint32_t box_word(uint32_t word, int w, const int lo[3], const int hi[3])
{
    const int lz = w >> 1;
    if (lz < lo[2] || lz >= hi[2])
        return 0u;
    const uint32_t xmask = ((1u << hi[0]) - 1u) & ~((1u << lo[0]) - 1u);
    uint32_t mask = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const int ly = (w & 1) * 4 + q;
        if (ly >= lo[1] && ly < hi[1])
            mask |= xmask << (q * 8);
    }
    return word & mask;
}

constexpr int kFaceThreads = 128; // face pass: one triangle per lane
constexpr int kRejectMin = 4;     // (triangle, brick) items with more candidates first test the whole box
constexpr int kFaceWindow = 512; // candidates listed per step of a warp
static_assert(kFaceWindow >= kBrick * kBrick * kBrick, "a dense item's candidates (up to a whole brick) fit the list");
static_assert(kFaceWindow >= kWordsPerBrick * 4, "the slot list holds a dense item's words");

struct FaceWarp
{
    float coef[kFaceCoef][32];         // face-test coefficients of each lane's triangle
    int info[11][32];                  // per lane: first brick (3), bricks along x and y, face box min (3), max (3)
    uint32_t pass[kWordsPerBrick][32]; // face-test hits of each item of the current chunk
    int org[3][32];                    // brick origin of each item
    uint8_t own[32];                   // lane whose triangle an item belongs to
    uint32_t tri[32];                  // triangle of each lane (global index)
    int seg[32];                       // mesh of each lane's triangle (batched conversions)
    uint16_t cl[kFaceWindow];          // candidate list: local voxel index
    alignas(16) uint8_t cs[kFaceWindow]; // candidate list: item slot (a dense item's 16 words while dense items run)
};

struct FaceCoefArr
{
    const float *c;
    __device__ __forceinline__ float operator()(int i) const
    {
        return c[i];
    }
};

struct FaceCoefSmem
{
    const float *p; // &coef[0][owner]
    __device__ __forceinline__ float operator()(int i) const
    {
        return p[i * 32];
    }
};

// Records of one (triangle, brick) item whose face-test hits are in column
// `lane` of pass (hits of them): COUNT adds them to the brick's record count
// and stages them (one reservation per warp; past the staging capacity they
// are only counted and the fill pass runs instead), FILL writes them into the
// brick's bucket.  Called by all lanes of the warp.
template <int M>
__device__ __forceinline__ void face_hits(const GenArgs &A, const uint32_t (*pass)[32], const int lane, const uint32_t hits,
                                          const long long b, const uint32_t tri)
{
    // COUNT: k0 is this item's first rank among brick b's records -- the scanline
    // records were all counted before, so it is the item's place in the bucket
    uint32_t k0 = 0;
    if (hits)
        k0 = agg_add(A.rcnt, b, hits);
    if (M == COUNT && A.fstage)
    {
        uint32_t incl = hits;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d)
                incl += y;
        }
        uint32_t base = 0;
        if (lane == 31 && incl)
            base = atomicAdd(&A.counters[C_FSTAGED], incl);
        base = __shfl_sync(0xffffffffu, base, 31);
        unsigned long long pos = (unsigned long long)base + incl - hits;
        uint32_t rank = k0;
        for (int w = 0; w < kWordsPerBrick && hits; ++w)
        {
            uint32_t pm = pass[w][lane];
            while (pm)
            {
                const int bt = __ffs(pm) - 1;
                pm &= pm - 1u;
                if (pos < A.fstage_cap)
                    A.fstage[pos] = make_uint4((uint32_t)b, tri, kRecFace | (uint32_t)(w * 32 + bt), rank);
                ++pos;
                ++rank;
            }
        }
    }
    if (M == FILL && hits)
    {
        if ((unsigned long long)k0 + hits > A.roff[b + 1] - A.roff[b])
            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_REPLAY);
        else
        {
            unsigned long long pos = A.roff[b] + k0;
            for (int w = 0; w < kWordsPerBrick; ++w)
            {
                uint32_t pm = pass[w][lane];
                while (pm)
                {
                    const int bt = __ffs(pm) - 1;
                    pm &= pm - 1u;
                    Rec rr;
                    rr.a = tri;
                    rr.b = kRecFace | (uint32_t)(w * 32 + bt);
                    rr.c = 0u;
                    A.rec[pos++] = rr;
                }
            }
        }
    }
}

// A lane's triangle in W: face-test coefficients, first brick and bricks along
// x and y of its face box, the face box itself, the triangle index.
__device__ __forceinline__ void face_lane_setup(FaceWarp &W, const int lane, const float v[3][3], const Grid &g, const int bmin[3],
                                                const int bmax[3], const int b0[3], const int nx, const int ny, const uint32_t t,
                                                const int sg)
{
    W.seg[lane] = sg;
    FaceSetup fs;
    face_setup(v, g, fs);
    float c[kFaceCoef];
    face_coefs(fs, c);
#pragma unroll
    for (int i = 0; i < kFaceCoef; ++i)
        W.coef[i][lane] = c[i];
    const int inf[11] = {b0[0], b0[1], b0[2], nx, ny, bmin[0], bmin[1], bmin[2], bmax[0], bmax[1], bmax[2]};
#pragma unroll
    for (int i = 0; i < 11; ++i)
        W.info[i][lane] = inf[i];
    W.tri[lane] = t;
}

// One round of (triangle, brick) items, one per lane: lane l's item is brick
// rank r of the face box of lane ol's triangle (coefficients, box and
// triangle in W at column ol).  The candidates (active voxels of the brick
// inside the face box) are tested on full warps: items with many of them by
// the whole warp with the coefficients in registers, the others through a
// shared list; then the hits become records.  Called by all lanes.
template <int M, bool B>
__device__ __forceinline__ void face_item(const GenArgs &A, FaceWarp &W, const int lane, const bool valid, const int ol, const int r)
{
    uint32_t cw[kWordsPerBrick];
    uint32_t cnt = 0;
    long long b = 0; // global brick of this lane's item
    if (valid)
    {
        const Mesh &Mi = mesh_of<B>(A, B ? W.seg[ol] : 0);
        const Grid &g = Mi.g;
        const int nx = W.info[3][ol], ny = W.info[4][ol];
        const int bx = W.info[0][ol] + r % nx, by = W.info[1][ol] + (r / nx) % ny, bz = W.info[2][ol] + r / (nx * ny);
        b = Mi.brick0 + (long long)bx + (long long)g.nb[0] * ((long long)by + (long long)g.nb[1] * (long long)bz);
        const int o[3] = {g.gmin[0] + bx * kBrick, g.gmin[1] + by * kBrick, g.gmin[2] + bz * kBrick};
        const int bmin[3] = {W.info[5][ol], W.info[6][ol], W.info[7][ol]};
        const int bmax[3] = {W.info[8][ol], W.info[9][ol], W.info[10][ol]};
        int lo[3], hi[3];
        const bool any = brick_box(bmin, bmax, o, lo, hi);
        const uint4 *bw4 = reinterpret_cast<const uint4 *>(A.bits + b * kWordsPerBrick);
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4)
        {
            const uint4 wv = any ? bw4[q4] : make_uint4(0u, 0u, 0u, 0u);
            const uint32_t words[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                cw[q4 * 4 + k] = any ? box_word(words[k], q4 * 4 + k, lo, hi) : 0u;
                cnt += __popc(cw[q4 * 4 + k]);
            }
        }
        if (cnt > (uint32_t)kRejectMin)
        {
            // the triangle misses the item's whole box: no candidate can pass
            const int alo[3] = {o[0] + lo[0], o[1] + lo[1], o[2] + lo[2]};
            const int ahi[3] = {o[0] + hi[0], o[1] + hi[1], o[2] + hi[2]};
            if (face_box_rejects(FaceCoefSmem{&W.coef[0][ol]}, g, alo, ahi))
            {
                cnt = 0;
#pragma unroll
                for (int w = 0; w < kWordsPerBrick; ++w)
                    cw[w] = 0u;
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
            W.org[a][lane] = o[a];
        W.own[lane] = (uint8_t)ol;
    }
    else
    {
#pragma unroll
        for (int w = 0; w < kWordsPerBrick; ++w)
            cw[w] = 0u;
    }
#pragma unroll
    for (int w = 0; w < kWordsPerBrick; ++w)
        W.pass[w][lane] = 0u;
    // items with many candidates are tested by the whole warp with the
    // triangle's coefficients in registers; the others go through the list
    const bool dense = cnt > (uint32_t)A.tune.dense_candidates;
    const uint32_t dmask = __ballot_sync(0xffffffffu, dense);
    __syncwarp();
    for (uint32_t dm = dmask; dm; dm &= dm - 1u)
    {
        // one dense item: its candidates are compacted into the shared list,
        // then tested by all lanes with the triangle's coefficients in registers
        const int sd = __ffs(dm) - 1;
        const int so = W.own[sd];
        float c[kFaceCoef];
#pragma unroll
        for (int i = 0; i < kFaceCoef; ++i)
            c[i] = W.coef[i][so];
        // this lane's half word of the item's candidates, passed on by the
        // item's lane through the slot list (unused while dense items run)
        uint32_t *dwords = reinterpret_cast<uint32_t *>(W.cs);
        if (lane == sd)
        {
#pragma unroll
            for (int ww = 0; ww < kWordsPerBrick; ++ww)
                dwords[ww] = cw[ww];
        }
        __syncwarp();
        const int w = lane >> 1;
        const uint32_t word = dwords[w];
        uint32_t bits = (lane & 1) ? (word & 0xffff0000u) : (word & 0x0000ffffu);
        uint32_t ntot;
        uint32_t pos = warp_exclusive_scan((uint32_t)__popc(bits), ntot);
        while (bits)
        {
            const int bt = __ffs(bits) - 1;
            bits &= bits - 1u;
            W.cl[pos++] = (uint16_t)(w * 32 + bt);
        }
        __syncwarp();
        const int ox = W.org[0][sd], oy = W.org[1][sd], oz = W.org[2][sd];
        const Grid &gd = mesh_of<B>(A, B ? W.seg[so] : 0).g;
        for (uint32_t k = lane; k < ntot; k += 32)
        {
            const int lv = W.cl[k];
            if (face_test_c(FaceCoefArr{c}, gd, ox + (lv & 7), oy + ((lv >> 3) & 7), oz + (lv >> 6)))
                atomicOr(&W.pass[lv >> 5][sd], 1u << (lv & 31));
        }
        __syncwarp();
    }
    const uint32_t lcnt = dense ? 0u : cnt;
    uint32_t off = lcnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, off, d);
        if (lane >= d)
            off += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, off, 31);
    off -= lcnt;
    for (uint32_t wbeg = 0; wbeg < total; wbeg += kFaceWindow)
    {
        // list the candidates that fall in [wbeg, wbeg + kFaceWindow)
        const uint32_t wend = wbeg + kFaceWindow;
        if (cnt && !dense && off < wend && off + cnt > wbeg)
        {
            uint32_t idx = off;
#pragma unroll 1
            for (int w = 0; w < kWordsPerBrick && idx < wend; ++w)
            {
                uint32_t word = cw[w];
                while (word && idx < wend)
                {
                    const int bt = __ffs(word) - 1;
                    word &= word - 1u;
                    if (idx >= wbeg)
                    {
                        W.cl[idx - wbeg] = (uint16_t)(w * 32 + bt);
                        W.cs[idx - wbeg] = (uint8_t)lane;
                    }
                    ++idx;
                }
            }
        }
        __syncwarp();
        const uint32_t n = total - wbeg < (uint32_t)kFaceWindow ? total - wbeg : (uint32_t)kFaceWindow;
        for (uint32_t k = lane; k < n; k += 32)
        {
            const int lv = W.cl[k], sl = W.cs[k];
            const int x = W.org[0][sl] + (lv & 7), y = W.org[1][sl] + ((lv >> 3) & 7), z = W.org[2][sl] + (lv >> 6);
            const Grid &gl = mesh_of<B>(A, B ? W.seg[W.own[sl]] : 0).g;
            if (face_test_c(FaceCoefSmem{&W.coef[0][W.own[sl]]}, gl, x, y, z))
                atomicOr(&W.pass[lv >> 5][sl], 1u << (lv & 31));
        }
        __syncwarp();
    }
    uint32_t hits = 0;
    if (cnt)
    {
#pragma unroll
        for (int w = 0; w < kWordsPerBrick; ++w)
            hits += __popc(W.pass[w][lane]);
    }
    face_hits<M>(A, W.pass, lane, hits, b, W.tri[ol]);
}

// Face stage (flexible_dual_grid.cpp:298-414), one triangle per lane.  The
// warp's (triangle, brick) items are taken 32 at a time; the candidates of
// those items (active voxels of the brick inside the triangle's face box) are
// listed in shared memory and tested by all 32 lanes, so the face tests run on
// full warps whatever the triangles' sizes.  COUNT adds each item's hits to its
// brick's record count; FILL writes one record per hit.
template <int M, typename IdxT, bool B>
__global__ void __launch_bounds__(kFaceThreads) face_records(GenArgs A)
{
    __shared__ FaceWarp FW[kFaceThreads / 32];
    const int lane = threadIdx.x & 31;
    FaceWarp &W = FW[threadIdx.x >> 5];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; // global triangle
    int nbk = 0;
    if (t < A.m.nf)
    {
        const int sg = seg_of_tri<B>(A, t);
        const Mesh &Ms = mesh_of<B>(A, sg);
        const Grid &g = Ms.g;
        float v[3][3];
        if (tri_load_m<B, IdxT>(Ms, t - Ms.tri0, v))
        {
            int bmin[3], bmax[3];
            face_box(v, g, bmin, bmax);
            if (bmax[0] > bmin[0] && bmax[1] > bmin[1] && bmax[2] > bmin[2])
            {
                int b0[3], b1[3];
#pragma unroll
                for (int a = 0; a < 3; ++a)
                {
                    b0[a] = (bmin[a] - g.gmin[a]) >> 3;
                    b1[a] = (bmax[a] - 1 - g.gmin[a]) >> 3;
                }
                const int nx = b1[0] - b0[0] + 1, ny = b1[1] - b0[1] + 1;
                const long long n = (long long)nx * ny * (b1[2] - b0[2] + 1);
                if (n > A.tune.inline_face_bricks)
                {
                    if (M == COUNT)
                    {
                        const uint32_t slot = atomicAdd(&A.counters[C_FACE_LARGE], 1u);
                        if (slot < A.face_large_cap)
                        {
                            A.face_large[slot] = (uint32_t)t;
                            A.face_units[slot] = (uint32_t)n;
                        }
                        else
                            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
                    }
                }
                else
                {
                    face_lane_setup(W, lane, v, g, bmin, bmax, b0, nx, ny, (uint32_t)t, sg);
                    nbk = (int)n;
                }
            }
        }
    }
    // items of the warp: exclusive scan of the lanes' brick counts
    int istart = nbk;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const int y = __shfl_up_sync(0xffffffffu, istart, d);
        if (lane >= d)
            istart += y;
    }
    const int nitems = __shfl_sync(0xffffffffu, istart, 31);
    istart -= nbk;
    __syncwarp();
    for (int ibase = 0; ibase < nitems; ibase += 32)
    {
        // item of this lane's slot: owner lane (last lane whose first item is at
        // or before it) and brick rank r within the owner's face box
        const int it = ibase + lane;
        int lo_l = 0;
#pragma unroll
        for (int step = 16; step >= 1; step >>= 1)
        {
            const int cand = lo_l + step;
            const int sv = __shfl_sync(0xffffffffu, istart, cand & 31);
            if (cand < 32 && sv <= it)
                lo_l = cand;
        }
        const int ol = lo_l;
        const int r = it - __shfl_sync(0xffffffffu, istart, ol);
        face_item<M, B>(A, W, lane, it < nitems, ol, r);
        __syncwarp();
    }
}

// Staged scanline records -> their bricks' buckets, through a cursor per brick.
__global__ void __launch_bounds__(kThreads) bucket_records(const uint4 *__restrict__ stage, uint32_t n, uint32_t *__restrict__ cursor,
                                                           const unsigned long long *__restrict__ roff, Rec *__restrict__ rec,
                                                           uint32_t *__restrict__ counters)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint4 r = stage[i];
    const long long b = (long long)r.x;
    const uint32_t k = agg_add(cursor, b, 1u);
    const unsigned long long base = roff[b];
    if (k >= roff[b + 1] - base)
    {
        atomicOr(&counters[C_STATUS], (uint32_t)ST_REPLAY);
        return;
    }
    Rec o;
    o.a = r.y;
    o.b = r.z;
    o.c = r.w;
    rec[base + k] = o;
}

// Triangles whose face box spans more than tune.inline_face_bricks bricks: their
// (triangle, brick) items, all listed triangles' items one after another, 32
// per warp and round, one per lane; the first lane of each run of a triangle's
// items sets the triangle up for the run, and the round runs as in
// face_records.  The grid is one resident wave; the warps loop over the units.
template <int M, typename IdxT, bool B>
__global__ void __launch_bounds__(kFaceThreads) large_faces(GenArgs A)
{
    __shared__ FaceWarp FW[kFaceThreads / 32];
    const int lane = threadIdx.x & 31;
    FaceWarp &W = FW[threadIdx.x >> 5];
    const uint32_t n = min(A.counters[C_FACE_LARGE], A.face_large_cap);
    const uint32_t total = A.counters[C_FUNITS];
    const int wpb = blockDim.x >> 5;
    const long long stride = (long long)gridDim.x * wpb * 32;
    for (long long ub = ((long long)blockIdx.x * wpb + (threadIdx.x >> 5)) * 32; ub < (long long)total; ub += stride)
    {
        const long long u = ub + lane;
        const bool inside = u < (long long)total;
        int r = 0;
        uint32_t i = 0xffffffffu;
        if (inside)
        {
            i = unit_owner(A.face_units, n, (uint32_t)u);
            r = (int)((uint32_t)u - A.face_units[i]);
        }
        // a triangle's items are consecutive: the first lane of each run sets
        // the triangle up once, the run's other lanes use that lane's column
        const uint32_t prev = __shfl_up_sync(0xffffffffu, i, 1);
        const bool first = inside && (lane == 0 || prev != i);
        const uint32_t firsts = __ballot_sync(0xffffffffu, first);
        const int ol = 31 - __clz(firsts & (0xffffffffu >> (31 - lane)));
        bool ok = false;
        if (first)
        {
            const uint32_t t = A.face_large[i];
            const int sg = seg_of_tri<B>(A, t);
            const Mesh &Ms = mesh_of<B>(A, sg);
            const Grid &g = Ms.g;
            float v[3][3];
            if (tri_load_m<B, IdxT>(Ms, t - Ms.tri0, v))
            {
                int bmin[3], bmax[3];
                face_box(v, g, bmin, bmax);
                int b0[3], b1[3];
#pragma unroll
                for (int a = 0; a < 3; ++a)
                {
                    b0[a] = (bmin[a] - g.gmin[a]) >> 3;
                    b1[a] = (bmax[a] - 1 - g.gmin[a]) >> 3;
                }
                face_lane_setup(W, lane, v, g, bmin, bmax, b0, b1[0] - b0[0] + 1, b1[1] - b0[1] + 1, t, sg);
                ok = true;
            }
        }
        const uint32_t oks = __ballot_sync(0xffffffffu, ok);
        const bool valid = inside && ((oks >> ol) & 1u);
        __syncwarp();
        face_item<M, B>(A, W, lane, valid, inside ? ol : lane, r);
        __syncwarp();
    }
}

// Staged face records -> their places in the bricks' buckets: the count pass
// staged each with its rank in the brick, so no cursor is needed.
__global__ void __launch_bounds__(kThreads) place_records(const uint4 *__restrict__ stage, uint32_t n,
                                                          const unsigned long long *__restrict__ roff, Rec *__restrict__ rec,
                                                          uint32_t *__restrict__ counters)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint4 r = stage[i];
    const long long b = (long long)r.x;
    const unsigned long long base = roff[b];
    if ((unsigned long long)r.w >= roff[b + 1] - base)
    {
        atomicOr(&counters[C_STATUS], (uint32_t)ST_REPLAY);
        return;
    }
    Rec o;
    o.a = r.y;
    o.b = r.z;
    o.c = 0u;
    rec[base + r.w] = o;
}

__global__ void copy_words(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[i];
}

constexpr int kLongWalk = 64; // boundary edges with a longer step bound are walked by a whole warp (default)

// One thread per boundary edge: the reference DDA walk; one record per active
// voxel visited.  Edges whose walk may take more than tune.long_walk steps are
// listed (COUNT) and left to boundary_long; FILL writes every edge's line
// quadric here.
template <int M, bool B>
__global__ void __launch_bounds__(kThreads) boundary_records(GenArgs A)
{
    const uint32_t n = min(A.counters[C_BOUNDARY], A.bkeys_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const unsigned long long e = A.bkeys[i];
        const uint32_t ia = (uint32_t)(e >> 32), ib = (uint32_t)(e & 0xffffffffull); // global vertex indices
        const Mesh &Ms = mesh_of<B>(A, seg_of_vert<B>(A, ia));
        const Grid &g = Ms.g;
        const uint32_t *bits = A.bits + Ms.brick0 * kWordsPerBrick;
        float v0[3], v1[3];
        vertex_load(Ms, ia - Ms.vert0, v0);
        vertex_load(Ms, ib - Ms.vert0, v1);
        Dda d;
        if (!boundary_setup(v0, v1, g, d, M == FILL ? A.btab + (size_t)i * 12 : nullptr))
            continue;
        if (d.guard > A.tune.long_walk)
        {
            if (M == COUNT)
            {
                const uint32_t slot = atomicAdd(&A.counters[C_BLONG], 1u);
                if (slot < A.blong_cap)
                    A.blong[slot] = i;
                else
                    atomicOr(&A.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
            }
            continue;
        }
        for (;;)
        {
            if (in_grid(g, d.cur[0], d.cur[1], d.cur[2]))
            {
                uint32_t bit;
                const long long w = voxel_word(g, d.cur[0], d.cur[1], d.cur[2], bit);
                if (bits[w] & (1u << bit))
                    put_record<M>(A, Ms.brick0 + (w >> 4), i, kRecBoundary | (uint32_t)((w & 15) * 32 + bit), 0u);
            }
            if (!dda_step(d))
                break;
        }
        if (d.guard < 0)
            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_WALK_GUARD);
    }
}

// The listed long boundary edges, one warp each.  Every lane runs the same
// DDA walk (the steps are cheap arithmetic); lane k visits steps k, k + 32,
// ..., so the occupancy lookups and records of 32 steps go out together.
template <int M, bool B>
__global__ void __launch_bounds__(kThreads) boundary_long(GenArgs A)
{
    const uint32_t n = min(A.counters[C_BLONG], A.blong_cap);
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (uint32_t j = blockIdx.x * wpb + (threadIdx.x >> 5); j < n; j += gridDim.x * wpb)
    {
        const uint32_t i = A.blong[j];
        const unsigned long long e = A.bkeys[i];
        const uint32_t ia = (uint32_t)(e >> 32), ib = (uint32_t)(e & 0xffffffffull); // global vertex indices
        const Mesh &Ms = mesh_of<B>(A, seg_of_vert<B>(A, ia));
        const Grid &g = Ms.g;
        const uint32_t *bits = A.bits + Ms.brick0 * kWordsPerBrick;
        float v0[3], v1[3];
        vertex_load(Ms, ia - Ms.vert0, v0);
        vertex_load(Ms, ib - Ms.vert0, v1);
        Dda d;
        if (!boundary_setup(v0, v1, g, d, nullptr))
            continue; // the same edge for the whole warp
        bool alive = true;
        while (alive)
        {
            int c[3] = {0, 0, 0};
            bool mine = false;
            for (int k = 0; k < 32 && alive; ++k)
            {
                if (k == lane)
                {
                    c[0] = d.cur[0];
                    c[1] = d.cur[1];
                    c[2] = d.cur[2];
                    mine = true;
                }
                alive = dda_step(d);
            }
            if (mine && in_grid(g, c[0], c[1], c[2]))
            {
                uint32_t bit;
                const long long w = voxel_word(g, c[0], c[1], c[2], bit);
                if (bits[w] & (1u << bit))
                    put_record<M>(A, Ms.brick0 + (w >> 4), i, kRecBoundary | (uint32_t)((w & 15) * 32 + bit), 0u);
            }
        }
        if (M == COUNT && lane == 0 && d.guard < 0)
            atomicOr(&A.counters[C_STATUS], (uint32_t)ST_WALK_GUARD);
    }
}

// ===========================================================================
// compaction and active-brick map
// ===========================================================================
__global__ void brick_count(const uint32_t *__restrict__ bits, long long nbricks, uint32_t *__restrict__ bcount,
                            uint32_t *__restrict__ aflag)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbricks)
        return;
    const uint4 *p = reinterpret_cast<const uint4 *>(bits + b * kWordsPerBrick);
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const uint4 q = p[i];
        c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
    }
    bcount[b] = c;
    aflag[b] = c ? 1u : 0u;
}

__global__ void brick_slots(const uint32_t *__restrict__ aflag, const unsigned long long *__restrict__ aslot, long long nbricks,
                            uint32_t *__restrict__ active)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbricks)
        return;
    if (aflag[b])
        active[aslot[b]] = (uint32_t)b;
}

// ===========================================================================
// boundary edges (edges used by exactly one face)
// ===========================================================================
template <typename IdxT>
__device__ __forceinline__ bool face_edge(const IdxT *faces, long long nv, long long f, int k, uint32_t &a, uint32_t &b)
{
    const long long i0 = (long long)faces[f * 3 + k], i1 = (long long)faces[f * 3 + (k + 1) % 3];
    const long long j0 = (long long)faces[f * 3 + (k + 2) % 3];
    if (i0 < 0 || i0 >= nv || i1 < 0 || i1 >= nv || j0 < 0 || j0 >= nv)
        return false;
    a = (uint32_t)(i0 < i1 ? i0 : i1);
    b = (uint32_t)(i0 < i1 ? i1 : i0);
    return true;
}

template <typename IdxT>
__global__ void edge_count(const IdxT *__restrict__ faces, long long nf, long long nv, uint32_t *__restrict__ vcnt)
{
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf)
        return;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        uint32_t a, b;
        if (face_edge(faces, nv, f, k, a, b))
            atomicAdd(&vcnt[a], 1u);
    }
}

template <typename IdxT>
__global__ void edge_fill(const IdxT *__restrict__ faces, long long nf, long long nv, const unsigned long long *__restrict__ voff,
                          uint32_t *__restrict__ vcnt, uint32_t *__restrict__ emax)
{
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf)
        return;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        uint32_t a, b;
        if (face_edge(faces, nv, f, k, a, b))
        {
            const uint32_t left = atomicSub(&vcnt[a], 1u);
            if (left == 0u)
                continue; // cannot happen: same faces as edge_count
            emax[voff[a] + (unsigned long long)(left - 1u)] = b;
        }
    }
}

// Edge k of global face f of a batched conversion, as global vertex indices.
__device__ __forceinline__ bool batch_face_edge(const Mesh *__restrict__ segs, int nseg, long long f, int k, uint32_t &a, uint32_t &b)
{
    const Mesh &M = segs[seg_find(nseg, f, [&](int i) { return segs[i].tri0; })];
    const long long fl = f - M.tri0;
    const bool ok = M.fbytes == 8 ? face_edge((const long long *)M.faces, M.nv, fl, k, a, b)
                                  : face_edge((const int *)M.faces, M.nv, fl, k, a, b);
    a += (uint32_t)M.vert0;
    b += (uint32_t)M.vert0;
    return ok;
}

__global__ void edge_count_batch(const Mesh *__restrict__ segs, int nseg, long long nf, uint32_t *__restrict__ vcnt)
{
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf)
        return;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        uint32_t a, b;
        if (batch_face_edge(segs, nseg, f, k, a, b))
            atomicAdd(&vcnt[a], 1u);
    }
}

__global__ void edge_fill_batch(const Mesh *__restrict__ segs, int nseg, long long nf, const unsigned long long *__restrict__ voff,
                                uint32_t *__restrict__ vcnt, uint32_t *__restrict__ emax)
{
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf)
        return;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        uint32_t a, b;
        if (batch_face_edge(segs, nseg, f, k, a, b))
        {
            const uint32_t left = atomicSub(&vcnt[a], 1u);
            if (left == 0u)
                continue; // cannot happen: same faces as edge_count_batch
            emax[voff[a] + (unsigned long long)(left - 1u)] = b;
        }
    }
}

__device__ void heap_sift(uint32_t *a, long long start, long long end)
{
    long long root = start;
    while (2 * root + 1 < end)
    {
        long long child = 2 * root + 1;
        if (child + 1 < end && a[child] < a[child + 1])
            ++child;
        if (a[root] < a[child])
        {
            const uint32_t t = a[root];
            a[root] = a[child];
            a[child] = t;
            root = child;
        }
        else
            return;
    }
}

// Sorts vertex a's list of larger endpoints (insertion sort for the usual
// short lists, heap sort beyond 32 entries).
__device__ void sort_list(uint32_t *l, long long n)
{
    if (n <= 32)
    {
        for (long long i = 1; i < n; ++i)
        {
            const uint32_t x = l[i];
            long long j = i;
            while (j > 0 && l[j - 1] > x)
            {
                l[j] = l[j - 1];
                --j;
            }
            l[j] = x;
        }
        return;
    }
    for (long long i = n / 2 - 1; i >= 0; --i)
        heap_sift(l, i, n);
    for (long long end = n - 1; end > 0; --end)
    {
        const uint32_t t = l[0];
        l[0] = l[end];
        l[end] = t;
        heap_sift(l, 0, end);
    }
}

// Per vertex a: sort the larger endpoints of the edges whose smaller endpoint
// is a and count those occurring once -- the boundary edges (a, b) (reference:
// std::map count == 1, flexible_dual_grid.cpp:741-757).
__global__ void edge_sort_count(const unsigned long long *__restrict__ voff, uint32_t *__restrict__ emax, long long nv,
                                uint32_t *__restrict__ bcnt)
{
    const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nv)
        return;
    const unsigned long long s = voff[a], e = voff[a + 1];
    const long long n = (long long)(e - s);
    uint32_t *l = emax + s;
    if (n <= 8)
    {
        // the usual case: the list in registers, Batcher's 19-comparator
        // network for 8 (padding sorts last: vertex indices are below 2^31)
        uint32_t r[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            r[i] = i < n ? l[i] : 0xffffffffu;
        constexpr int net[19][2] = {{0, 1}, {2, 3}, {4, 5}, {6, 7}, {0, 2}, {1, 3}, {4, 6}, {5, 7}, {1, 2}, {5, 6},
                                    {0, 4}, {1, 5}, {2, 6}, {3, 7}, {2, 4}, {3, 5}, {1, 2}, {3, 4}, {5, 6}};
#pragma unroll
        for (int k = 0; k < 19; ++k)
        {
            const uint32_t x = r[net[k][0]], y = r[net[k][1]];
            r[net[k][0]] = min(x, y);
            r[net[k][1]] = max(x, y);
        }
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (i < n)
            {
                l[i] = r[i];
                const bool dup = (i > 0 && r[i - 1] == r[i]) || (i + 1 < n && r[i + 1] == r[i]);
                c += dup ? 0u : 1u;
            }
        bcnt[a] = c;
        return;
    }
    sort_list(l, n);
    uint32_t c = 0;
    for (long long i = 0; i < n;)
    {
        long long j = i;
        while (j < n && l[j] == l[i])
            ++j;
        c += (j - i == 1);
        i = j;
    }
    bcnt[a] = c;
}

// Per vertex a: its boundary edges at their rank in (a, b) order, so the
// boundary list is sorted like the reference's std::map.
__global__ void edge_emit(const unsigned long long *__restrict__ voff, const uint32_t *__restrict__ emax, long long nv,
                          const unsigned long long *__restrict__ boff, unsigned long long *__restrict__ bkeys,
                          unsigned long long bkeys_cap, uint32_t *__restrict__ counters)
{
    const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nv)
        return;
    const unsigned long long s = voff[a], e = voff[a + 1];
    const long long n = (long long)(e - s);
    const uint32_t *l = emax + s;
    unsigned long long k = boff[a];
    for (long long i = 0; i < n;)
    {
        long long j = i;
        while (j < n && l[j] == l[i])
            ++j;
        if (j - i == 1)
        {
            if (k < bkeys_cap)
                bkeys[k] = ((unsigned long long)a << 32) | l[i];
            else
                atomicOr(&counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
            ++k;
        }
        i = j;
    }
}

// ===========================================================================
// per-brick accumulation in reference order + solve
// ===========================================================================
struct SolveArgs
{
    Mesh m;
    const Mesh *segs; // batched conversions: the meshes (global memory)
    int nseg;
    float bw, rw;
    const uint32_t *bits;
    const unsigned long long *bbase;
    const uint32_t *active;
    const unsigned long long *roff;
    const Rec *rec;
    const float *qtab;
    const float *btab;
    int32_t *vox;
    float *dual;
    uint8_t *flags;
    uint32_t *counters;
    uint2 *contrib;             // per-voxel contribution lists {order key, payload}
    unsigned long long contrib_cap; // entries contrib holds
    uint32_t key_face, key_boundary; // first face and boundary order keys: 12F and 13F
    bool zorder;                // output rows in z-order (bbase then holds z-order row bases)
    uint32_t *longv;            // rows whose lists are too long for voxel_accumulate: up to kLongMidMax
                                // entries from the front (counter C_LONG), longer ones from the back (C_HUGE)
    uint32_t longv_cap;
    unsigned long long *vlist;  // per output row: first contribution (low 40 bits) | count << 40 | sorted << 63
    float *clist; // deferred constrained searches, 16 words each (full: searched inline)
    uint32_t clist_cap;
    float route_tol; // compensated precision: FP32 solve error (voxel edges) above which a voxel is solved in FP64
};

// Rank of active voxel lv among the brick's voxels in output order.
template <typename SS>
__device__ __forceinline__ int dense_index(const SS &S, int lv)
{
    const int r = S.zorder ? local_morton(lv) : lv;
    const int w = r >> 5, b = r & 31;
    return (int)(S.wpre[w] + __popc(S.bits[w] & ((1u << b) - 1u)));
}

// Loads a brick's occupancy into S (obits, bits in output-rank order, wpre,
// nvox); the calling CTA must not use S before the final barrier.
template <typename SS>
__device__ __forceinline__ void load_brick_ranks(SS &S, const uint32_t *__restrict__ bits, long long b, bool zorder)
{
    const int tid = threadIdx.x;
    if (tid < kWordsPerBrick)
    {
        const uint32_t w = bits[b * kWordsPerBrick + tid];
        S.obits[tid] = w;
        S.bits[tid] = zorder ? 0u : w;
    }
    if (tid == 0)
        S.zorder = zorder ? 1 : 0;
    __syncthreads();
    if (zorder)
    {
        for (int lv = tid; lv < 512; lv += blockDim.x)
            if ((S.obits[lv >> 5] >> (lv & 31)) & 1u)
            {
                const int m = local_morton(lv);
                atomicOr(&S.bits[m >> 5], 1u << (m & 31));
            }
        __syncthreads();
    }
    if (tid < 32)
    {
        const uint32_t w = tid < kWordsPerBrick ? S.bits[tid] : 0u;
        const uint32_t c = __popc(w);
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (tid >= d)
                incl += y;
        }
        if (tid < kWordsPerBrick)
            S.wpre[tid] = incl - c;
        if (tid == 31)
            S.nvox = (int)incl;
    }
    __syncthreads();
}

// Expand one record of the brick into (dense voxel index, order key, payload)
// contributions; key_face and key_boundary are 12F and 13F.
template <typename SS, typename Sink>
__device__ __forceinline__ void expand(const SS &S, const Rec &r, uint32_t key_face, uint32_t key_boundary, Sink &sink)
{
    const uint32_t kind = r.b >> 30;
    if (kind == 0)
    {
        const int ax2 = (int)(r.b & 3u);
        const int u = (int)((r.b >> 2) & 15u) - 1, v = (int)((r.b >> 6) & 15u) - 1, w = (int)((r.b >> 10) & 15u);
        const uint32_t kb = (r.a * 3u + (uint32_t)ax2) * 4u;
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            const int dx = k >> 1, dy = k & 1;
            const int lu = u + dx, lv = v + dy;
            if (lu < 0 || lu >= 8 || lv < 0 || lv >= 8)
                continue;
            int lx, ly, lz;
            place(ax2, lu, lv, w, lx, ly, lz);
            sink(dense_index(S, lx + 8 * ly + 64 * lz), kb + (uint32_t)((1 - dy) * 2 + (1 - dx)), r.c);
        }
    }
    else if (kind == 1)
        sink(dense_index(S, (int)(r.b & 511u)), key_face + r.a, 0u);
    else
        sink(dense_index(S, (int)(r.b & 511u)), key_boundary + r.a, 0u);
}

struct Acc
{
    float q[10];
    float mean[3];
    float cnt;
    uint32_t flags;
    bool first;
};

__device__ __forceinline__ void acc_init(Acc &a)
{
#pragma unroll
    for (int i = 0; i < 10; ++i)
        a.q[i] = 0.0f;
    a.mean[0] = a.mean[1] = a.mean[2] = 0.0f;
    a.cnt = 0.0f;
    a.flags = 0;
    a.first = true;
}

// One contribution decoded and loaded, ready to be added (flexible_dual_grid.cpp:251-271, :409, :521).
struct Contrib
{
    float q[10];
    float p[3];
    uint32_t flag;
    unsigned stage;
};

// A quadric of a 12-float (48-byte) table row: three 16-byte loads.
__device__ __forceinline__ void load_q12(const float *p, float q[10])
{
    const float4 a = reinterpret_cast<const float4 *>(p)[0], b = reinterpret_cast<const float4 *>(p)[1];
    const float2 c = reinterpret_cast<const float2 *>(p)[4];
    q[0] = a.x; q[1] = a.y; q[2] = a.z; q[3] = a.w;
    q[4] = b.x; q[5] = b.y; q[6] = b.z; q[7] = b.w;
    q[8] = c.x; q[9] = c.y;
}

__device__ __forceinline__ void contrib_load(const SolveArgs &A, const Grid &g, const int vc[3], uint32_t key, uint32_t pay,
                                             Contrib &c)
{
    c.stage = key < A.key_face ? 0u : (key < A.key_boundary ? 1u : 2u);
    c.flag = 0u;
    c.p[0] = c.p[1] = c.p[2] = 0.0f;
    if (c.stage == 0)
    {
        const uint32_t ta = key >> 2;
        const uint32_t t = ta / 3u;
        const int ax2 = (int)(ta - t * 3u);
        const int dx = 1 - (int)(key & 1u), dy = 1 - (int)((key >> 1) & 1u);
        const int ax0 = (ax2 + 1) % 3, ax1 = (ax2 + 2) % 3;
        const int c0 = ax0 == 0 ? vc[0] : (ax0 == 1 ? vc[1] : vc[2]);
        const int c1 = ax1 == 0 ? vc[0] : (ax1 == 1 ? vc[1] : vc[2]);
        const float vs0 = ax0 == 0 ? g.vs[0] : (ax0 == 1 ? g.vs[1] : g.vs[2]);
        const float vs1 = ax1 == 0 ? g.vs[0] : (ax1 == 1 ? g.vs[1] : g.vs[2]);
        const float pu = (float)(c0 - dx + 1) * vs0;
        const float pv = (float)(c1 - dy + 1) * vs1;
        const float pw = __uint_as_float(pay);
        c.p[0] = ax2 == 0 ? pw : (ax2 == 1 ? pv : pu);
        c.p[1] = ax2 == 0 ? pu : (ax2 == 1 ? pw : pv);
        c.p[2] = ax2 == 0 ? pv : (ax2 == 1 ? pu : pw);
        load_q12(A.qtab + (size_t)t * 12, c.q);
        if (dx == 0 && dy == 0)
            c.flag = 1u << ax2;
    }
    else if (c.stage == 1)
        load_q12(A.qtab + (size_t)(key - A.key_face) * 12, c.q);
    else
    {
        // line quadric of boundary edge e (computed once by the boundary pass), weighted
        float bq[10];
        load_q12(A.btab + (size_t)(key - A.key_boundary) * 12, bq);
#pragma unroll
        for (int i = 0; i < 10; ++i)
            c.q[i] = A.bw * bq[i];
    }
}

// Adds one contribution in reference order; the first one is copied (keeps signed zeros).
__device__ __forceinline__ void contrib_apply(const Contrib &c, Acc &a)
{
    if (c.stage == 0)
    {
        if (a.first)
        {
            a.mean[0] = c.p[0];
            a.mean[1] = c.p[1];
            a.mean[2] = c.p[2];
            a.cnt = 1.0f;
#pragma unroll
            for (int i = 0; i < 10; ++i)
                a.q[i] = c.q[i];
            a.first = false;
        }
        else
        {
            a.mean[0] = a.mean[0] + c.p[0];
            a.mean[1] = a.mean[1] + c.p[1];
            a.mean[2] = a.mean[2] + c.p[2];
            a.cnt = a.cnt + 1.0f;
#pragma unroll
            for (int i = 0; i < 10; ++i)
                a.q[i] = a.q[i] + c.q[i];
        }
        a.flags |= c.flag;
    }
    else
    {
#pragma unroll
        for (int i = 0; i < 10; ++i)
            a.q[i] = a.q[i] + c.q[i];
    }
}

// ---------------------------------------------------------------------------
// Contribution lists: one CTA per active brick expands the brick's records
// and counting-sorts the contributions by voxel into global memory (the
// brick reserves exactly its entries with one atomic on counters[C_CONTRIB];
// the total, four per scanline event and one per other record, sized the
// buffer); then one thread per voxel orders its list by key, sums it in that
// order (the reference CPU order) and solves.
// ---------------------------------------------------------------------------
// Order key of a contribution list entry {key, payload}.
__device__ __forceinline__ uint32_t entry_key(const uint2 &e)
{
    return e.x;
}

struct ListShared
{
    uint32_t obits[kWordsPerBrick]; // occupancy words (bit = local index)
    uint32_t bits[kWordsPerBrick];  // the same voxels in output-rank order (z-order: bit = local z-order rank)
    uint32_t wpre[kWordsPerBrick];  // prefix counts of bits
    int zorder;
    uint32_t cnt[512];
    uint32_t off[512];
    uint32_t scan_tmp[kConsumeThreads / 32 + 1]; // per-warp offsets, then the brick's total
    int nvox;
    uint32_t status;
    unsigned long long first; // the brick's first contribution entry (reserved by one atomic)
    // the brick's lists, when they fit (keys and payloads apart): filled,
    // short lists sorted, copied out
    uint32_t skey[kListStage];
    uint32_t spay[kListStage];
};

struct ListCount
{
    ListShared &S;
    __device__ __forceinline__ void operator()(int i, uint32_t, uint32_t) const
    {
        atomicAdd(&S.cnt[i], 1u);
    }
};

struct ListFill
{
    ListShared &S;
    uint2 *out;    // the brick's first entry
    uint32_t room; // entries the brick reserved
    __device__ __forceinline__ void operator()(int i, uint32_t key, uint32_t pay) const
    {
        // off[i] counts up from the start of voxel i's list: records are taken
        // in bucket order, which is close to key order, so lists come out nearly sorted
        const uint32_t k = atomicAdd(&S.off[i], 1u);
        if (k >= room)
        {
            atomicOr(&S.status, (uint32_t)ST_REPLAY);
            return;
        }
        out[k] = make_uint2(key, pay);
    }
};

// The same into the brick's shared staging arrays.
struct ListStageFill
{
    ListShared &S;
    __device__ __forceinline__ void operator()(int i, uint32_t key, uint32_t pay) const
    {
        const uint32_t k = atomicAdd(&S.off[i], 1u);
        if (k >= (uint32_t)kListStage)
        {
            atomicOr(&S.status, (uint32_t)ST_REPLAY);
            return;
        }
        S.skey[k] = key;
        S.spay[k] = pay;
    }
};

template <bool B>
__global__ void __launch_bounds__(kConsumeThreads) brick_lists(SolveArgs A)
{
    __shared__ ListShared S;
    const int tid = threadIdx.x;
    const long long b = A.active[blockIdx.x]; // global brick
    int o[3];
    {
        const Mesh &Ms = mesh_of<B>(A, seg_of_brick<B>(A, b));
        brick_origin(Ms.g, b - Ms.brick0, o);
    }
    const Rec *rec = A.rec + A.roff[b];
    const unsigned long long nrec = A.roff[b + 1] - A.roff[b];
    for (int i = tid; i < 512; i += blockDim.x)
        S.cnt[i] = 0;
    if (tid == 0)
        S.status = 0;
    load_brick_ranks(S, A.bits, b, A.zorder);
    const int nvox = S.nvox;
    const unsigned long long vbase = A.bbase[b];
    // voxel coordinates of the brick's rows (every thread a quarter of the brick)
    for (int lv = tid; lv < 512; lv += blockDim.x)
    {
        if ((S.obits[lv >> 5] >> (lv & 31)) & 1u)
        {
            const long long row = (long long)(vbase + dense_index(S, lv));
            A.vox[row * 3 + 0] = o[0] + (lv & 7);
            A.vox[row * 3 + 1] = o[1] + ((lv >> 3) & 7);
            A.vox[row * 3 + 2] = o[2] + (lv >> 6);
        }
    }
    {
        ListCount cs{S};
        for (unsigned long long r = tid; r < nrec; r += blockDim.x)
            expand(S, rec[r], A.key_face, A.key_boundary, cs);
    }
    __syncthreads();
    // exclusive scan of the counts: off[i] = start of voxel i's list
    {
        const int lane = tid & 31, warp = tid >> 5;
        constexpr int per = 512 / kConsumeThreads;
        uint32_t v[per], sum = 0;
#pragma unroll
        for (int k = 0; k < per; ++k)
        {
            const int j = tid * per + k;
            v[k] = j < nvox ? S.cnt[j] : 0u;
            sum += v[k];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d)
                incl += y;
        }
        if (lane == 31)
            S.scan_tmp[warp] = incl;
        __syncthreads();
        if (tid == 0)
        {
            uint32_t r = 0;
            for (int k = 0; k < kConsumeThreads / 32; ++k)
            {
                const uint32_t x = S.scan_tmp[k];
                S.scan_tmp[k] = r;
                r += x;
            }
            S.scan_tmp[kConsumeThreads / 32] = r;
            // the brick's room in contrib: exactly its entries
            unsigned long long f = atomicAdd((unsigned long long *)&A.counters[C_CONTRIB], (unsigned long long)r);
            if (f + r > A.contrib_cap)
            {
                atomicOr(&S.status, (uint32_t)ST_LIST_OVERFLOW);
                f = ~0ull;
            }
            S.first = f;
        }
        __syncthreads();
        if (S.first == ~0ull)
        {
            if (tid == 0)
                atomicOr(&A.counters[C_STATUS], S.status);
            return;
        }
        const bool staged = S.scan_tmp[kConsumeThreads / 32] <= (uint32_t)kListStage;
        uint32_t run = S.scan_tmp[warp] + incl - sum;
        const unsigned long long first = S.first;
#pragma unroll
        for (int k = 0; k < per; ++k)
        {
            const int j = tid * per + k;
            if (j < nvox)
            {
                if (v[k] == 0u || v[k] > kListCountMax)
                    atomicOr(&S.status, (uint32_t)ST_REPLAY); // every active voxel has a scanline contribution
                const bool sorted = staged && v[k] < (uint32_t)kWarpSortMin;
                A.vlist[vbase + j] = (first + run) | ((unsigned long long)v[k] << 40) | (sorted ? kListSorted : 0ull);
            }
            S.off[j] = run;
            run += v[k];
        }
    }
    __syncthreads();
    const uint32_t total = S.scan_tmp[kConsumeThreads / 32];
    uint2 *out = A.contrib + S.first;
    if (total <= (uint32_t)kListStage)
    {
        // the lists fit in shared memory: fill them there, sort the short ones
        // (one thread per voxel), copy the brick's lists out in one sweep
        {
            ListStageFill fs{S};
            for (unsigned long long r = tid; r < nrec; r += blockDim.x)
                expand(S, rec[r], A.key_face, A.key_boundary, fs);
        }
        __syncthreads();
        for (int j = tid; j < nvox; j += blockDim.x)
        {
            const uint32_t c = S.cnt[j];
            if (c < 2u || c >= (uint32_t)kWarpSortMin)
                continue;
            uint32_t *K = S.skey + (S.off[j] - c);
            uint32_t *P = S.spay + (S.off[j] - c);
            for (uint32_t x = 1; x < c; ++x)
            {
                const uint32_t k = K[x];
                const uint32_t pv = P[x];
                uint32_t y = x;
                while (y > 0 && K[y - 1] > k)
                {
                    K[y] = K[y - 1];
                    P[y] = P[y - 1];
                    --y;
                }
                K[y] = k;
                P[y] = pv;
            }
        }
        __syncthreads();
        for (uint32_t i = tid; i < total; i += blockDim.x)
            out[i] = make_uint2(S.skey[i], S.spay[i]);
    }
    else
    {
        ListFill fs{S, out, total};
        for (unsigned long long r = tid; r < nrec; r += blockDim.x)
            expand(S, rec[r], A.key_face, A.key_boundary, fs);
    }
    __syncthreads();
    if (tid == 0 && S.status)
        atomicOr(&A.counters[C_STATUS], S.status);
}

// One thread per voxel row: order the voxel's contributions by key, sum them in
// that order, regularise and solve (flexible_dual_grid.cpp:763-797); voxels
// whose unconstrained solution leaves the box go to the constrained-search list.

// Regularise and solve one voxel (flexible_dual_grid.cpp:763-797); a voxel whose
// unconstrained solution leaves its box goes to the constrained-search list.
// Compensated sums (precision mode "compensated"): each of the 14 running sums
// (quadric, mass point, count) keeps its float value and the float error of
// its additions (Knuth's TwoSum, exact without contraction), merged in double
// at the end.
struct AccC
{
    float s[14], e[14];
    uint32_t flags;
};

__device__ __forceinline__ void acc_init(AccC &a)
{
#pragma unroll
    for (int i = 0; i < 14; ++i)
        a.s[i] = a.e[i] = 0.0f;
    a.flags = 0;
}

__device__ __forceinline__ void two_sum_add(float &s, float &e, float x)
{
    const float t = s + x;
    const float bp = t - s;
    e = e + ((s - (t - bp)) + (x - bp));
    s = t;
}

__device__ __forceinline__ void contrib_apply(const Contrib &c, AccC &a)
{
#pragma unroll
    for (int i = 0; i < 10; ++i)
        two_sum_add(a.s[i], a.e[i], c.q[i]);
    if (c.stage == 0)
    {
#pragma unroll
        for (int i = 0; i < 3; ++i)
            two_sum_add(a.s[10 + i], a.e[10 + i], c.p[i]);
        two_sum_add(a.s[13], a.e[13], 1.0f);
        a.flags |= c.flag;
    }
}

__device__ __forceinline__ void voxel_finish(const SolveArgs &A, const Grid &g, long long row, const int vc[3], const Acc &a);

// The constrained search for a voxel the full deferred list could not take:
// a call of its own, so that its registers stay out of the accumulate loop.
// Everything is passed by value (taking the address of the kernel's
// parameters would move them to local memory); the search uses only the
// grid's voxel size.
struct Q10
{
    float v[10];
};

__device__ __noinline__ void constrained_here(float *dual, long long row, int x, int y, int z, float vx, float vy, float vz, Q10 q)
{
    Grid g{};
    g.vs[0] = vx;
    g.vs[1] = vy;
    g.vs[2] = vz;
    const int vc[3] = {x, y, z};
    float w[3];
    solve_constrained(vc, g, q.v, w);
    dual[row * 3 + 0] = w[0];
    dual[row * 3 + 1] = w[1];
    dual[row * 3 + 2] = w[2];
}

// Compensated precision: sums merged and regularised in double; the FP32
// solve of the rounded quadric is kept unless its error estimate -- the
// pivoted QR's condition estimate |R00|/|R22| times FLT_EPSILON times the
// voxel's distance from the grid origin in voxel edges -- exceeds
// A.route_tol voxel edges, in which case the voxel is solved (and, if
// needed, box-constrained) in double.
__device__ __forceinline__ void voxel_finish(const SolveArgs &A, const Grid &g, long long row, const int vc[3], const AccC &a)
{
    double qd[10], md[3];
#pragma unroll
    for (int i = 0; i < 10; ++i)
        qd[i] = (double)a.s[i] + (double)a.e[i];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        md[i] = (double)a.s[10 + i] + (double)a.e[10 + i];
    const double cd = (double)a.s[13] + (double)a.e[13];
    double qr[10];
    regularize_t<double>(qd, md, cd, (double)A.rw, qr);
    A.flags[row * 3 + 0] = (uint8_t)(a.flags & 1u);
    A.flags[row * 3 + 1] = (uint8_t)((a.flags >> 1) & 1u);
    A.flags[row * 3 + 2] = (uint8_t)((a.flags >> 2) & 1u);
    float qf[10];
#pragma unroll
    for (int i = 0; i < 10; ++i)
        qf[i] = (float)qr[i];
    float v[3], rd[3];
    const bool inside = solve_unconstrained_t<float>(vc, g, qf, v, rd);
    float ext = 1.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        ext = fmaxf(ext, fabsf((float)vc[i]) + 1.0f);
    const float r0 = fabsf(rd[0]), r2 = fabsf(rd[2]);
    if (!(r2 > 0.0f) || (r0 / r2) * FLT_EPSILON * ext > A.route_tol)
    {
        atomicAdd(&A.counters[C_ROUTED], 1u);
        double vd[3];
        if (!solve_unconstrained_t<double>(vc, g, qr, vd))
            solve_constrained_t<double>(vc, g, qr, vd);
        A.dual[row * 3 + 0] = (float)vd[0];
        A.dual[row * 3 + 1] = (float)vd[1];
        A.dual[row * 3 + 2] = (float)vd[2];
        return;
    }
    if (inside)
    {
        A.dual[row * 3 + 0] = v[0];
        A.dual[row * 3 + 1] = v[1];
        A.dual[row * 3 + 2] = v[2];
        return;
    }
    const uint32_t slot = atomicAdd(&A.counters[C_CONSTRAINED], 1u);
    if (slot >= A.clist_cap)
    {
        // the deferred list is full: search here (same routine, same result)
        Q10 qv;
#pragma unroll
        for (int i = 0; i < 10; ++i)
            qv.v[i] = qf[i];
        constrained_here(A.dual, row, vc[0], vc[1], vc[2], g.vs[0], g.vs[1], g.vs[2], qv);
        return;
    }
    float *c = A.clist + (size_t)slot * 16;
    c[0] = __int_as_float((int)row);
    c[1] = __int_as_float(vc[0]);
    c[2] = __int_as_float(vc[1]);
    c[3] = __int_as_float(vc[2]);
#pragma unroll
    for (int i = 0; i < 10; ++i)
        c[4 + i] = qf[i];
}

__device__ __forceinline__ void voxel_finish(const SolveArgs &A, const Grid &g, long long row, const int vc[3], const Acc &a)
{
    float q[10];
    regularize(a.q, a.mean, a.cnt, A.rw, q);
    float v[3];
    const bool inside = solve_unconstrained(vc, g, q, v);
    A.flags[row * 3 + 0] = (uint8_t)(a.flags & 1u);
    A.flags[row * 3 + 1] = (uint8_t)((a.flags >> 1) & 1u);
    A.flags[row * 3 + 2] = (uint8_t)((a.flags >> 2) & 1u);
    if (inside)
    {
        A.dual[row * 3 + 0] = v[0];
        A.dual[row * 3 + 1] = v[1];
        A.dual[row * 3 + 2] = v[2];
        return;
    }
    const uint32_t slot = atomicAdd(&A.counters[C_CONSTRAINED], 1u);
    if (slot >= A.clist_cap)
    {
        // the deferred list is full: search here (same routine, same result)
        Q10 qv;
#pragma unroll
        for (int i = 0; i < 10; ++i)
            qv.v[i] = q[i];
        constrained_here(A.dual, row, vc[0], vc[1], vc[2], g.vs[0], g.vs[1], g.vs[2], qv);
        return;
    }
    float *c = A.clist + (size_t)slot * 16;
    c[0] = __int_as_float((int)row);
    c[1] = __int_as_float(vc[0]);
    c[2] = __int_as_float(vc[1]);
    c[3] = __int_as_float(vc[2]);
#pragma unroll
    for (int i = 0; i < 10; ++i)
        c[4 + i] = q[i];
}

constexpr int kWarpSortPer = 2;                      // ... up to 2 entries per lane
constexpr int kWarpSortMax = 32 * kWarpSortPer;      // longer lists go to voxel_accumulate_long
constexpr int kLongMidMax = 1024;                    // ... one CTA of 128 threads, shared-memory sort
constexpr int kLongHugeMax = 8192;                   // ... one CTA of 256 threads; longer: in-place insertion sort

// 12 resident CTAs per SM (at most 40 registers): the sums wait on gathers,
// and the extra warps hide more of that than the few spills cost; the
// compensated-precision variant, with twice the running sums and an FP64
// solve, gets 4 (128 registers)
template <bool B, int P>
__global__ void __launch_bounds__(128, P == 0 ? 12 : 4) voxel_accumulate(SolveArgs A, long long nrows)
{
    const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = row < nrows;
    const unsigned long long d = valid ? A.vlist[row] : 0ull;
    const unsigned long long first = d & ((1ull << 40) - 1ull);
    const uint32_t n = (uint32_t)(d >> 40) & kListCountMax;
    const bool sorted = (d & kListSorted) != 0ull;
    // The warp orders the longer lists of its 32 voxels one after another: each
    // lane holds up to kWarpSortPer entries of the list and finds their ranks
    // among the list's (unique) keys, then stores the entries at those ranks.
    const uint32_t need = __ballot_sync(0xffffffffu, n >= (uint32_t)kWarpSortMin && n <= (uint32_t)kWarpSortMax);
    for (uint32_t m = need; m; m &= m - 1u)
    {
        const int v = __ffs(m) - 1;
        const uint32_t nv = __shfl_sync(0xffffffffu, n, v);
        const unsigned long long fv = __shfl_sync(0xffffffffu, first, v);
        uint2 *L = A.contrib + fv;
        const uint2 pad = make_uint2(0xffffffffu, 0u);
        uint2 e[kWarpSortPer];
        uint32_t k[kWarpSortPer];
        uint32_t r[kWarpSortPer];
#pragma unroll
        for (int q = 0; q < kWarpSortPer; ++q)
        {
            const uint32_t idx = (uint32_t)(lane + 32 * q);
            e[q] = idx < nv ? L[idx] : pad;
            k[q] = entry_key(e[q]);
            r[q] = 0;
        }
        // rank = number of smaller keys (keys are unique per voxel; ties, which
        // cannot occur, would keep list order)
#pragma unroll
        for (int sq = 0; sq < kWarpSortPer; ++sq)
        {
            if ((uint32_t)(32 * sq) >= nv)
                break;
            const uint32_t jn = nv - 32u * sq < 32u ? nv - 32u * sq : 32u;
            for (uint32_t j = 0; j < jn; ++j)
            {
                const uint32_t kj = __shfl_sync(0xffffffffu, k[sq], (int)j);
                const uint32_t jj = 32u * sq + j;
#pragma unroll
                for (int q = 0; q < kWarpSortPer; ++q)
                    r[q] += kj < k[q] || (kj == k[q] && jj < (uint32_t)(lane + 32 * q));
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < kWarpSortPer; ++q)
            if ((uint32_t)(lane + 32 * q) < nv)
                L[r[q]] = e[q];
    }
    __syncwarp();
    if (!valid)
        return;
    if (n > (uint32_t)kWarpSortMax)
    {
        // long list: left to voxel_accumulate_long (one CTA per voxel)
        const bool huge = n > (uint32_t)kLongMidMax;
        const uint32_t slot = atomicAdd(&A.counters[huge ? C_HUGE : C_LONG], 1u);
        if (slot < A.longv_cap)
        {
            A.longv[huge ? A.longv_cap - 1u - slot : slot] = (uint32_t)row;
            return;
        }
        atomicOr(&A.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
        return;
    }
    const int vc[3] = {A.vox[row * 3 + 0], A.vox[row * 3 + 1], A.vox[row * 3 + 2]};
    const Grid &g = mesh_of<B>(A, seg_of_row<B>(A, row)).g;
    uint2 *lst = A.contrib + first;
    if (n < (uint32_t)kWarpSortMin && !sorted)
    {
        // short lists that brick_lists could not sort in shared memory:
        // insertion sort in place
        for (uint32_t x = 1; x < n; ++x)
        {
            const uint2 e = lst[x];
            const uint32_t k = entry_key(e);
            uint32_t j = x;
            while (j > 0)
            {
                const uint2 pe = lst[j - 1];
                if (entry_key(pe) <= k)
                    break;
                lst[j] = pe;
                --j;
            }
            if (j != x)
                lst[j] = e;
        }
    }
    std::conditional_t<P == 0, Acc, AccC> a;
    acc_init(a);
    for (uint32_t x = 0; x < n; ++x)
    {
        const uint2 e = lst[x];
        Contrib c;
        contrib_load(A, g, vc, entry_key(e), e.y, c);
        contrib_apply(c, a);
    }
    voxel_finish(A, g, row, vc, a);
}

constexpr int kLongChunk = 256; // contributions staged per step of the sequential sum
template <int kMax>
constexpr size_t long_smem()
{
    return (size_t)kMax * 8 + (size_t)kLongChunk * sizeof(Contrib);
}

// One CTA per voxel with a long contribution list (coarse grids over dense
// meshes): bitonic sort of the keys in shared memory, then the contributions
// are loaded by all threads a chunk at a time and summed in order by one
// thread.  Lists longer than kMax are insertion-sorted in place (slow,
// correct).
// kHuge = false: lists of up to kLongMidMax entries (front of longv); true: longer lists (back of longv).
template <int kMax, int kThreadsT, bool kHuge, bool B, int P>
__global__ void __launch_bounds__(kThreadsT) voxel_accumulate_long(SolveArgs A)
{
    extern __shared__ uint4 lsm[];
    uint32_t *key = reinterpret_cast<uint32_t *>(lsm);
    uint32_t *pay = key + kMax;
    Contrib *cb = reinterpret_cast<Contrib *>(pay + kMax);
    const int tid = threadIdx.x;
    const uint32_t nlong = min(A.counters[kHuge ? C_HUGE : C_LONG], A.longv_cap);
    for (uint32_t li = blockIdx.x; li < nlong; li += gridDim.x)
    {
        const long long row = A.longv[kHuge ? A.longv_cap - 1u - li : li];
        const unsigned long long d = A.vlist[row];
        const unsigned long long first = d & ((1ull << 40) - 1ull);
        const uint32_t n = (uint32_t)(d >> 40) & kListCountMax;
        const int vc[3] = {A.vox[row * 3 + 0], A.vox[row * 3 + 1], A.vox[row * 3 + 2]};
        const Grid &g = mesh_of<B>(A, seg_of_row<B>(A, row)).g;
        uint2 *lst = A.contrib + first;
        std::conditional_t<P == 0, Acc, AccC> a;
        acc_init(a);
        if (n <= (uint32_t)kMax)
        {
            uint32_t p2 = 1;
            while (p2 < n)
                p2 <<= 1;
            for (uint32_t i = tid; i < p2; i += blockDim.x)
            {
                if (i < n)
                {
                    const uint2 e = lst[i];
                    key[i] = entry_key(e);
                    pay[i] = e.y;
                }
                else
                {
                    key[i] = ~0u;
                    pay[i] = 0u;
                }
            }
            __syncthreads();
            for (uint32_t k = 2; k <= p2; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1)
                {
                    for (uint32_t i = tid; i < p2; i += blockDim.x)
                    {
                        const uint32_t l = i ^ j;
                        if (l > i)
                        {
                            const bool up = (i & k) == 0;
                            const uint32_t ki = key[i], kl = key[l];
                            if ((ki > kl) == up)
                            {
                                key[i] = kl;
                                key[l] = ki;
                                const uint32_t t = pay[i];
                                pay[i] = pay[l];
                                pay[l] = t;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t c0 = 0; c0 < n; c0 += kLongChunk)
            {
                const uint32_t cn = min((uint32_t)kLongChunk, n - c0);
                for (uint32_t i = tid; i < cn; i += blockDim.x)
                    contrib_load(A, g, vc, key[c0 + i], pay[c0 + i], cb[i]);
                __syncthreads();
                if (tid == 0)
                    for (uint32_t i = 0; i < cn; ++i)
                        contrib_apply(cb[i], a);
                __syncthreads();
            }
        }
        else if (tid == 0)
        {
            for (uint32_t x = 1; x < n; ++x)
            {
                const uint2 e = lst[x];
                const uint32_t k = entry_key(e);
                uint32_t j = x;
                while (j > 0)
                {
                    const uint2 pe = lst[j - 1];
                    if (entry_key(pe) <= k)
                        break;
                    lst[j] = pe;
                    --j;
                }
                if (j != x)
                    lst[j] = e;
            }
            for (uint32_t x = 0; x < n; ++x)
            {
                const uint2 e = lst[x];
                Contrib c;
                contrib_load(A, g, vc, entry_key(e), e.y, c);
                contrib_apply(c, a);
            }
        }
        if (tid == 0)
            voxel_finish(A, g, row, vc, a);
        __syncthreads();
    }
}

// Constrained search (faces, edges, corners of the voxel box) for the voxels
// whose unconstrained solution left the box; one thread per listed voxel.
template <bool B>
__global__ void __launch_bounds__(128) constrained_solve(const float *__restrict__ clist, const uint32_t *__restrict__ counters,
                                                         uint32_t cap, Grid g1, const Mesh *__restrict__ segs, int nseg,
                                                         float *__restrict__ dual)
{
    const uint32_t n = min(counters[C_CONSTRAINED], cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float *c = clist + (size_t)i * 16;
        const long long row = __float_as_int(c[0]);
        const int vc[3] = {__float_as_int(c[1]), __float_as_int(c[2]), __float_as_int(c[3])};
        float q[10];
#pragma unroll
        for (int k = 0; k < 10; ++k)
            q[k] = c[4 + k];
        float v[3];
        if constexpr (B)
            solve_constrained(vc, segs[seg_find(nseg, row, [&](int s) { return segs[s].row0; })].g, q, v);
        else
            solve_constrained(vc, g1, q, v);
        dual[row * 3 + 0] = v[0];
        dual[row * 3 + 1] = v[1];
        dual[row * 3 + 2] = v[2];
    }
}

// Occupancy only: coordinates of every active voxel, one CTA per active brick.
struct CoordShared
{
    uint32_t obits[kWordsPerBrick];
    uint32_t bits[kWordsPerBrick];
    uint32_t wpre[kWordsPerBrick];
    int zorder;
    int nvox;
};

// Coordinates of the active voxels (intersect_occ output), one CTA per active brick.
__global__ void __launch_bounds__(128) brick_coords(const uint32_t *__restrict__ bits, const unsigned long long *__restrict__ bbase,
                                                    const uint32_t *__restrict__ active, Grid g, bool zorder, int32_t *__restrict__ vox)
{
    __shared__ CoordShared S;
    const long long b = active[blockIdx.x];
    load_brick_ranks(S, bits, b, zorder);
    int o[3];
    brick_origin(g, b, o);
    const unsigned long long base = bbase[b];
    for (int lv = threadIdx.x; lv < 512; lv += blockDim.x)
    {
        if (!((S.obits[lv >> 5] >> (lv & 31)) & 1u))
            continue;
        const long long row = (long long)(base + dense_index(S, lv));
        vox[row * 3 + 0] = o[0] + (lv & 7);
        vox[row * 3 + 1] = o[1] + ((lv >> 3) & 7);
        vox[row * 3 + 2] = o[2] + (lv >> 6);
    }
}

// z-order row bases: sort key of each active brick (its z-order code) ...
// In a batched conversion the key leads with the brick's mesh (bits 42 and up),
// so that each mesh's rows stay together, in z-order inside the mesh (brick
// coordinates below 2^14 per axis).
template <bool B>
__global__ void zorder_brick_keys(const uint32_t *__restrict__ active, long long n_active, Grid g1, const Mesh *__restrict__ segs,
                                  int nseg, unsigned long long *__restrict__ keys, uint32_t *__restrict__ slots)
{
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_active)
        return;
    long long b = active[s];
    unsigned long long lead = 0;
    const Grid *gp = &g1;
    if constexpr (B)
    {
        const int sg = seg_find(nseg, b, [&](int i) { return segs[i].brick0; });
        b -= segs[sg].brick0;
        gp = &segs[sg].g;
        lead = (unsigned long long)sg << 42;
    }
    const Grid &g = *gp;
    const unsigned long long bx = (unsigned long long)(g.gmin[0] / kBrick) + (unsigned long long)(b % g.nb[0]);
    const unsigned long long by = (unsigned long long)(g.gmin[1] / kBrick) + (unsigned long long)((b / g.nb[0]) % g.nb[1]);
    const unsigned long long bz = (unsigned long long)(g.gmin[2] / kBrick) + (unsigned long long)(b / ((long long)g.nb[0] * g.nb[1]));
    keys[s] = lead | brick_morton(bx, by, bz);
    slots[s] = (uint32_t)s;
}

// ... voxel counts in that order ...
__global__ void zorder_counts(const uint32_t *__restrict__ sorted_slots, long long n_active, const uint32_t *__restrict__ active,
                              const uint32_t *__restrict__ bcount, uint32_t *__restrict__ cnt)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n_active)
        cnt[j] = bcount[active[sorted_slots[j]]];
    else if (j == n_active)
        cnt[j] = 0u;
}

// ... and their exclusive scan scattered back to the bricks.
__global__ void zorder_bases(const uint32_t *__restrict__ sorted_slots, long long n_active, const uint32_t *__restrict__ active,
                             const unsigned long long *__restrict__ base_sorted, unsigned long long *__restrict__ zbase)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n_active)
        zbase[active[sorted_slots[j]]] = base_sorted[j];
}

// .vxz attribute packing of a conversion's outputs (examples/mesh2ovox.py:51-54):
// dual vertex -> clamp(dual * res - coord, 0, 1) * 255 truncated to uint8, one
// operation at a time in float32 as there; flags -> x + 2y + 4z in one byte.
__global__ void fdg_pack_kernel(const int32_t *__restrict__ vox, const float *__restrict__ dual, const uint8_t *__restrict__ inter,
                                long long n, float r0, float r1, float r2, uint8_t *__restrict__ dual_u8, uint8_t *__restrict__ inter_u8)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float r[3] = {r0, r1, r2};
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        float d = __fsub_rn(__fmul_rn(dual[i * 3 + a], r[a]), (float)vox[i * 3 + a]);
        d = fminf(fmaxf(d, 0.0f), 1.0f);
        dual_u8[i * 3 + a] = (uint8_t)(int)__fmul_rn(d, 255.0f);
    }
    inter_u8[i] = (uint8_t)((inter[i * 3 + 0] ? 1 : 0) + 2 * (inter[i * 3 + 1] ? 1 : 0) + 4 * (inter[i * 3 + 2] ? 1 : 0));
}

// o_voxel.serialize z-order codes (serialize/z_order.cu:33-97): 10 bits per coordinate.
__global__ void z_order_encode_kernel(const int32_t *__restrict__ x, const int32_t *__restrict__ y, const int32_t *__restrict__ z,
                                      long long n, int32_t *__restrict__ codes)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t c = (spread3_10((uint32_t)x[i] & 1023u) << 2) | (spread3_10((uint32_t)y[i] & 1023u) << 1) |
                       spread3_10((uint32_t)z[i] & 1023u);
    codes[i] = (int32_t)c;
}

__global__ void z_order_decode_kernel(const int32_t *__restrict__ codes, long long n, int32_t *__restrict__ x,
                                      int32_t *__restrict__ y, int32_t *__restrict__ z)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t c = (uint32_t)codes[i];
    x[i] = (int32_t)compact3_10(c >> 2);
    y[i] = (int32_t)compact3_10(c >> 1);
    z[i] = (int32_t)compact3_10(c);
}

// Hilbert codes (o_voxel.serialize mode 'hilbert', src/serialize/hilbert.cu:33-130):
// J. Skilling's transposed Hilbert index ("Programming the Hilbert curve",
// AIP Conf. Proc. 707, 2004) for 3 axes of 10 bits, its three transposed words
// interleaved like the z-order code.  One thread per code; the bit planes are
// walked with the axes in registers.
__device__ __forceinline__ void hilbert_exchange(uint32_t &a0, uint32_t &ai, uint32_t q)
{
    const uint32_t low = q - 1u;
    if (ai & q)
        a0 ^= low;
    else
    {
        const uint32_t swap = (a0 ^ ai) & low;
        a0 ^= swap;
        ai ^= swap;
    }
}

__global__ void hilbert_encode_kernel(const int32_t *__restrict__ x, const int32_t *__restrict__ y, const int32_t *__restrict__ z,
                                      long long n, int32_t *__restrict__ codes)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint32_t a0 = (uint32_t)x[i] & 1023u, a1 = (uint32_t)y[i] & 1023u, a2 = (uint32_t)z[i] & 1023u;
    // undo the excess work, top bit plane first
#pragma unroll
    for (uint32_t q = 1u << 9; q > 1u; q >>= 1)
    {
        hilbert_exchange(a0, a0, q);
        hilbert_exchange(a0, a1, q);
        hilbert_exchange(a0, a2, q);
    }
    // Gray encode
    a1 ^= a0;
    a2 ^= a1;
    uint32_t flip = 0;
#pragma unroll
    for (uint32_t q = 1u << 9; q > 1u; q >>= 1)
        if (a2 & q)
            flip ^= q - 1u;
    a0 ^= flip;
    a1 ^= flip;
    a2 ^= flip;
    codes[i] = (int32_t)((spread3_10(a0) << 2) | (spread3_10(a1) << 1) | spread3_10(a2));
}

__global__ void hilbert_decode_kernel(const int32_t *__restrict__ codes, long long n, int32_t *__restrict__ x,
                                      int32_t *__restrict__ y, int32_t *__restrict__ z)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t c = (uint32_t)codes[i];
    uint32_t a0 = compact3_10(c >> 2), a1 = compact3_10(c >> 1), a2 = compact3_10(c);
    // Gray decode
    const uint32_t half = a2 >> 1;
    a2 ^= a1;
    a1 ^= a0;
    a0 ^= half;
    // redo the excess work, bottom bit plane first
#pragma unroll
    for (uint32_t q = 2u; q != (1u << 10); q <<= 1)
    {
        hilbert_exchange(a0, a2, q);
        hilbert_exchange(a0, a1, q);
        hilbert_exchange(a0, a0, q);
    }
    x[i] = (int32_t)a0;
    y[i] = (int32_t)a1;
    z[i] = (int32_t)a2;
}

// ===========================================================================
// allocation-free occupancy (ovx_fdg_occupancy_noalloc)
// ===========================================================================
// All scratch of this entry point lives in one file-scope device array: the
// occupancy bitmap of up to kNoallocMaxBricks bricks, then one 32-bit row base
// per brick plus the total.  Every call shares it; each call clears the bitmap
// it uses before marking.
constexpr long long kNoallocMaxBricks = 32768; // e.g. a 256^3 grid
constexpr size_t kNoallocBitsBytes = (size_t)kNoallocMaxBricks * kWordsPerBrick * 4;
constexpr size_t kNoallocBytes = kNoallocBitsBytes + (size_t)(kNoallocMaxBricks + 1) * 4;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

__global__ void noalloc_clear(uint32_t *__restrict__ bits, long long words)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (long long)gridDim.x * blockDim.x)
        bits[i] = 0u;
}

// Scanline occupancy of a triangle soup, one thread per (triangle, axis), every row inline.
__global__ void __launch_bounds__(kThreads) noalloc_mark(const float *__restrict__ tris, long long nt, Grid g, uint32_t *bits)
{
    const long long ta = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (ta >= 3 * nt)
        return;
    const long long t = ta / 3;
    const int ax2 = (int)(ta - 3 * t);
    float v[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            v[k][c] = tris[t * 9 + k * 3 + c];
    AxisScan s;
    axis_setup(v, ax2, g, s);
    auto sink = [&](int xi, int yi, int zi, float, float, double) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
        {
            int x, y, z;
            place(ax2, xi + (k >> 1), yi + (k & 1), zi, x, y, z);
            uint32_t bit;
            const long long w = voxel_word(g, x, y, z, bit);
            atomicOr(&bits[w], 1u << bit);
        }
    };
#pragma unroll 1
    for (int yi = s.start; yi < s.end; ++yi)
        scan_row(s, yi, INT_MIN, INT_MAX, g, sink);
}

// One CTA: popcount per brick and exclusive scan into row bases; base[nb] = total.
__global__ void __launch_bounds__(1024) noalloc_scan(const uint32_t *__restrict__ bits, long long nb, uint32_t *__restrict__ base)
{
    __shared__ uint32_t warp_sum[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long per = (nb + blockDim.x - 1) / blockDim.x;
    const long long b0 = (long long)tid * per;
    const long long b1 = b0 + per < nb ? b0 + per : nb;
    uint32_t local = 0;
    for (long long b = b0; b < b1; ++b)
        for (int w = 0; w < kWordsPerBrick; ++w)
            local += __popc(bits[b * kWordsPerBrick + w]);
    uint32_t incl = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d)
            incl += y;
    }
    if (lane == 31)
        warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t ws = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d)
                wi += y;
        }
        if (lane < (int)(blockDim.x >> 5))
            warp_sum[lane] = wi - ws;
        if (lane == (int)(blockDim.x >> 5) - 1)
            base[nb] = wi;
    }
    __syncthreads();
    uint32_t run = warp_sum[warp] + incl - local;
    for (long long b = b0; b < b1; ++b)
    {
        base[b] = run;
        for (int w = 0; w < kWordsPerBrick; ++w)
            run += __popc(bits[b * kWordsPerBrick + w]);
    }
}

// One thread per occupancy word: coordinates of its voxels at their rows (brick order).
__global__ void noalloc_emit(const uint32_t *__restrict__ bits, const uint32_t *__restrict__ base, Grid g, int32_t *__restrict__ vox)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nbricks * kWordsPerBrick)
        return;
    uint32_t word = bits[i];
    if (!word)
        return;
    const long long b = i / kWordsPerBrick;
    const int w = (int)(i - b * kWordsPerBrick);
    uint32_t row = base[b];
    for (int k = 0; k < w; ++k)
        row += __popc(bits[b * kWordsPerBrick + k]);
    int o[3];
    brick_origin(g, b, o);
    while (word)
    {
        const int bt = __ffs(word) - 1;
        word &= word - 1u;
        const int lv = w * 32 + bt;
        vox[(long long)row * 3 + 0] = o[0] + (lv & 7);
        vox[(long long)row * 3 + 1] = o[1] + ((lv >> 3) & 7);
        vox[(long long)row * 3 + 2] = o[2] + (lv >> 6);
        ++row;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// Stage timers: CUDA events recorded at these points when profiling is on.
enum
{
    EV_BEGIN = 0,
    EV_EVENTS_COUNT,
    EV_COMPACT,
    EV_EDGES,
    EV_RECORD_COUNT,
    EV_FINISH,
    EV_EVENTS_FILL,
    EV_RECORD_FILL,
    EV_CONSUME,
    EV_SOLVE,
    EV_CONSTRAINED,
    kStageEvents
};
const char *const kStageNames[] = {"scanline_mark_count", "compaction", "boundary_edges", "face_boundary_count",
                                   "scanline_fill", "face_boundary_fill", "brick_lists", "voxel_accumulate",
                                   "constrained_solve"};
constexpr int kStages = 9;

struct Buf
{
    void *p = nullptr;
    size_t cap = 0;
};

} // namespace

struct ovx_fdg_context
{
    int device = 0;
    int sms = 148;
    Buf bits, bcount, bbase, aflag, aslot, active, counters, scan_large, scan_units, face_large, face_units, qtab;
    Buf vcnt, voff, emax, bkeys, blong, boff, btab;
    Buf rcnt, roff, rec, cub_tmp, cub_tmp_side, vlist, longv, face_end;
    Buf arena; // staged event records, then staged face records; after the fills, the contribution lists
    Buf zkeys, zslots, zcnt, zsbase, zbase; // z-order row bases
    Buf unit_tiles;                         // tile sums of the unit-list scans
    Buf segs_d;                             // batched conversion: the meshes (device copy of segs)
    std::vector<Mesh> segs;                 // batched conversion: the meshes, with their global offsets
    Mesh *segs_pinned = nullptr;            // staging of the mesh table for its upload (pinned)
    unsigned long long *seg_rows = nullptr; // first output row of every mesh and the total: pinned, mapped
    unsigned long long *seg_rows_dev = nullptr;
    int seg_cap = 0;                        // meshes the pinned buffers hold
    bool batch = false;                     // the conversion in progress is a batched one
    Tuning tune{kUnitCells, kWarpScanWork, kInlineFaceBricks, kDenseCandidates, kLongWalk};
    int precision = 0;       // OVX_FDG_PRECISION_*
    float route_tol = 1e-3f; // compensated precision: FP32 solve error estimate (voxel edges) that routes a voxel to FP64
    unsigned long long *host = nullptr;     // readback words: pinned, mapped host memory
    unsigned long long *host_dev = nullptr; // the same words as the device addresses them
    cudaMemPool_t pool = nullptr;       // workspace pool (keeps its memory until the context is destroyed)
    std::string err;
    // state between begin and finish
    int phase = 0; // 0 idle, 1 after begin (full), 2 after begin (occupancy only)
    Grid g{};
    const float *verts = nullptr;
    long long nv = 0;
    const void *faces = nullptr;
    int fbytes = 4;
    long long nf = 0;
    float origin[3] = {0, 0, 0};
    float fw = 0, bw = 0, rw = 0;
    long long n_vox = 0, n_active = 0, n_rec = 0, n_boundary = 0;
    unsigned long long n_lunits = 0, n_funits = 0, n_blong = 0; // large-pair and large-face units, long boundary edges
    unsigned long long n_fstaged = 0, fstage_want = 0; // face records staged by the count pass (and the most seen)
    bool face_staged = false;                         // all of them fitted: the fill pass need not redo the tests
    unsigned long long n_estaged = 0, estage_want = 0; // the same for the scanline event records
    bool event_staged = false;
    unsigned long long estage_n = 0, fstage_n = 0; // staging room in the arena: event records, then face records
    unsigned long long n_events = 0, n_contrib = 0; // scanline events; contribution entries (4 per event, 1 per other record)
    int order = 0;                                    // output row order: 0 brick-linear, 1 z-order
    int finished = 0;
    long long launches = 0; // kernels this library launched (its own, not CUB's)
    bool profiling = false;
    cudaEvent_t ev[kStageEvents] = {};
    // end of the last conversion's queued work: the next conversion, possibly
    // on another stream, waits for it before reusing the workspace
    cudaEvent_t done = nullptr;
    // second stream of begin: the boundary-edge pipeline runs on it beside the scanline pass
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool done_valid = false;
    bool grew = false; // a buffer grew during this conversion: the pool gives back what it no longer backs
    // work lists of begin (large pairs, large triangles, long boundary edges,
    // boundary edges): sized from the most entries seen, else a guess; a
    // conversion whose lists overflow runs its begin once more with exact sizes
    unsigned long long want_scan = 0, want_face = 0, want_blong = 0, want_bkeys = 0;
    unsigned long long list_guess = 65536; // floor of the guess (tests set OVX_FDG_LIST_GUESS)
    long long clist_limit = -1; // entries of the deferred constrained list (-1: as many as fit; tests set
                                // OVX_FDG_CLIST_LIMIT to send voxels down the inline path)
};

namespace
{

template <typename Ctx>
int buffer_list(Ctx *c, Buf **out)
{
    Buf *b[] = {&c->bits, &c->bcount, &c->bbase, &c->aflag, &c->aslot, &c->active, &c->counters, &c->scan_large, &c->scan_units,
                &c->face_large, &c->face_units, &c->qtab, &c->vcnt, &c->voff, &c->emax, &c->bkeys, &c->blong, &c->boff, &c->btab, &c->rcnt, &c->roff, &c->rec,
                &c->cub_tmp, &c->cub_tmp_side, &c->vlist, &c->arena, &c->longv, &c->face_end,
                &c->zkeys, &c->zslots, &c->zcnt, &c->zsbase, &c->zbase, &c->segs_d, &c->unit_tiles};
    const int n = (int)(sizeof(b) / sizeof(b[0]));
    for (int i = 0; i < n; ++i)
        out[i] = b[i];
    return n;
}

void stage(ovx_fdg_context *c, int i, cudaStream_t st)
{
    if (c->profiling && c->ev[i])
        cudaEventRecord(c->ev[i], st);
}

// Orders this call after the context's previous conversion, whatever its stream.
cudaError_t wait_previous(ovx_fdg_context *c, cudaStream_t st)
{
    if (!c->done_valid)
        return cudaSuccess;
    return cudaStreamWaitEvent(st, c->done, 0);
}

cudaError_t mark_done(ovx_fdg_context *c, cudaStream_t st)
{
    if (!c->done)
    {
        const cudaError_t e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
        if (e != cudaSuccess)
            return e;
    }
    const cudaError_t e = cudaEventRecord(c->done, st);
    c->done_valid = e == cudaSuccess;
    return e;
}

int fail(ovx_fdg_context *c, int status, const char *what)
{
    if (c)
        c->err = what;
    return status;
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

int cuda_fail(ovx_fdg_context *c, cudaError_t e, const char *where)
{
    if (c)
    {
        c->err = std::string(where) + ": " + cudaGetErrorString(e);
        c->phase = 0;
    }
    return e == cudaErrorMemoryAllocation ? OVX_FDG_OUT_OF_MEMORY : OVX_FDG_CUDA_ERROR;
}

#define OVX_CUDA(call)                                   \
    do                                                   \
    {                                                    \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess)                           \
            return cuda_fail(ctx, e_, #call);            \
    } while (0)

// Grows a workspace buffer in stream order from the context's own memory pool:
// the old block goes back to the pool behind the work queued on `st`, and no
// call here waits for the device, so contexts converting on other streams
// (the batched API's workers) are not stalled when one of them grows.
cudaError_t ensure(cudaStream_t st, ovx_fdg_context *ctx, Buf &b, size_t bytes)
{
    if (bytes == 0)
        bytes = 16;
    if (b.cap >= bytes)
        return cudaSuccess;
    if (b.p)
    {
        cudaFreeAsync(b.p, st);
        b.p = nullptr;
        b.cap = 0;
    }
    const size_t want = bytes + bytes / 8 + 256;
    ctx->grew = true;
    cudaError_t e = cudaMallocFromPoolAsync(&b.p, want, ctx->pool, st);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        b.p = nullptr;
        return e;
    }
    b.cap = want;
    return cudaSuccess;
}

// Exclusive scan with CUB; `tmp` is the scratch of the stream it runs on.
template <typename In, typename Out>
cudaError_t exclusive_scan(ovx_fdg_context *ctx, const In *in, Out *out, long long n, cudaStream_t st, Buf *tmp = nullptr)
{
    Buf &t = tmp ? *tmp : ctx->cub_tmp;
    size_t bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveScan(nullptr, bytes, in, out, cub::Sum(), Out(0), (int)n, st);
    if (e != cudaSuccess)
        return e;
    e = ensure(st, ctx, t, bytes);
    if (e != cudaSuccess)
        return e;
    return cub::DeviceScan::ExclusiveScan(t.p, bytes, in, out, cub::Sum(), Out(0), (int)n, st);
}

// The context's second stream and its fork/join events, created on first use.
cudaError_t side_stream(ovx_fdg_context *ctx)
{
    cudaError_t e = cudaSuccess;
    if (!ctx->side)
        e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->fork_ev)
        e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->join_ev)
        e = cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming);
    return e;
}

inline unsigned blocks_for(long long n, int threads)
{
    return (unsigned)((n + threads - 1) / threads);
}

// z-order row bases of the active bricks (ctx->zbase, indexed by brick): the
// bricks' z-order codes sorted, their voxel counts scanned in that order.
int zorder_row_bases(ovx_fdg_context *ctx, cudaStream_t st)
{
    const long long na = ctx->n_active, nb = ctx->g.nbricks;
    OVX_CUDA(ensure(st, ctx, ctx->zkeys, (size_t)(na + 1) * 16));
    OVX_CUDA(ensure(st, ctx, ctx->zslots, (size_t)(na + 1) * 8));
    OVX_CUDA(ensure(st, ctx, ctx->zcnt, (size_t)(na + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->zsbase, (size_t)(na + 1) * 8));
    OVX_CUDA(ensure(st, ctx, ctx->zbase, (size_t)(nb + 1) * 8));
    if (na == 0)
        return OVX_FDG_OK;
    unsigned long long *kin = (unsigned long long *)ctx->zkeys.p, *kout = kin + (na + 1);
    uint32_t *vin = (uint32_t *)ctx->zslots.p, *vout = vin + (na + 1);
    const uint32_t *active = (const uint32_t *)ctx->active.p;
    int end_bit = 63;
    if (ctx->batch)
        zorder_brick_keys<true><<<blocks_for(na, 256), 256, 0, st>>>(active, na, ctx->g, (const Mesh *)ctx->segs_d.p,
                                                                     (int)ctx->segs.size(), kin, vin);
    else
    {
        zorder_brick_keys<false><<<blocks_for(na, 256), 256, 0, st>>>(active, na, ctx->g, nullptr, 0, kin, vin);
        // key bits: 3 x (bits of the largest brick coordinate)
        int cb = 1;
        for (int a = 0; a < 3; ++a)
        {
            const long long mx = ctx->g.gmin[a] / kBrick + ctx->g.nb[a];
            while ((1ll << cb) <= mx)
                ++cb;
        }
        end_bit = std::min(63, 3 * cb);
    }
    size_t bytes = 0;
    OVX_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, (int)na, 0, end_bit, st));
    OVX_CUDA(ensure(st, ctx, ctx->cub_tmp, bytes));
    OVX_CUDA(cub::DeviceRadixSort::SortPairs(ctx->cub_tmp.p, bytes, kin, kout, vin, vout, (int)na, 0, end_bit, st));
    zorder_counts<<<blocks_for(na + 1, 256), 256, 0, st>>>(vout, na, active, (const uint32_t *)ctx->bcount.p,
                                                          (uint32_t *)ctx->zcnt.p);
    OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->zcnt.p, (unsigned long long *)ctx->zsbase.p, na + 1, st));
    zorder_bases<<<blocks_for(na, 256), 256, 0, st>>>(vout, na, active, (const unsigned long long *)ctx->zsbase.p,
                                                     (unsigned long long *)ctx->zbase.p);
    ctx->launches += 3;
    OVX_CUDA(cudaGetLastError());
    return OVX_FDG_OK;
}


int check_grid(ovx_fdg_context *ctx, const ovx_fdg_grid *grid, Grid &g)
{
    if (!grid)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "grid is NULL");
    long long nb = 1;
    for (int a = 0; a < 3; ++a)
    {
        const float vs = grid->voxel_size[a];
        if (!(vs > 0.0f) || !(vs < 3.0e38f))
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "voxel_size must be positive and finite");
        g.vs[a] = vs;
        g.rv[a] = 1.0 / (double)vs;
        g.gmin[a] = grid->grid_min[a];
        g.gmax[a] = grid->grid_max[a];
        const long long sz = (long long)grid->grid_max[a] - (long long)grid->grid_min[a];
        if (sz < 1 || sz > (1 << 20))
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "grid_range must satisfy 1 <= grid_max - grid_min <= 2^20");
        g.size[a] = (int)sz;
        g.nb[a] = (int)((sz + kBrick - 1) / kBrick);
        nb *= g.nb[a];
    }
    if (ctx->order == 1)
        for (int a = 0; a < 3; ++a)
            if (g.gmin[a] < 0 || g.gmin[a] % kBrick != 0)
                return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "z-order output needs grid_min >= 0 and a multiple of 8 on every axis");
    if (nb * kWordsPerBrick * 4ll > (64ll << 30) || nb >= (1ll << 31))
        return fail(ctx, OVX_FDG_CAPACITY, "grid too large for the dense brick bitmap (64 GiB limit)");
    g.nbricks = nb;
    return OVX_FDG_OK;
}

Mesh make_mesh(const ovx_fdg_context *c)
{
    Mesh m{};
    m.g = c->g;
    m.verts = c->verts;
    m.nv = c->nv;
    m.faces = c->faces;
    m.nf = c->nf;
    m.ox = c->origin[0];
    m.oy = c->origin[1];
    m.oz = c->origin[2];
    m.fbytes = c->fbytes;
    return m;
}

// Host readback words of a context: [0] rows, [1] active bricks, [2] records,
// [kHostCounters..] the counters after begin, [kHostFinish..] after finish.
constexpr int kHostCounters = 4;
constexpr int kHostFinish = 16;
constexpr int kHostWords = 32;
static_assert(kHostCounters * 8 + C_WORDS * 4 <= kHostFinish * 8 && kHostFinish * 8 + C_WORDS * 4 <= kHostWords * 8,
              "readback regions overlap");

__global__ void copy_word(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst)
{
    *dst = *src;
}

// First output row of every mesh of a batched conversion, into the mesh table
// (row0) and into mapped host memory, then the total.
__global__ void seg_rows(Mesh *__restrict__ segs, int nseg, const unsigned long long *__restrict__ bbase, long long nb,
                         unsigned long long *host)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    volatile unsigned long long *h = host;
    if (i < nseg)
    {
        const unsigned long long r = bbase[segs[i].brick0];
        segs[i].row0 = (long long)r;
        h[i] = r;
    }
    else if (i == nseg)
        h[i] = bbase[nb];
    __threadfence_system();
}

// The mesh table of a batched conversion, from mapped host memory (a kernel
// rather than a copy, which could queue behind another stream's large copy).
__global__ void load_segs(const uint32_t *__restrict__ src, uint32_t *__restrict__ dst, long long words)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (long long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

// Up to kReadbackMax device words/blocks to copy into the mapped readback
// words.  Adding more sets `overflow`, which the caller turns into an
// OVX_FDG_INTERNAL error before launching (a dropped entry would leave a stale
// host word to be read as a count).
constexpr int kReadbackMax = 4;
struct Readback
{
    const void *src[kReadbackMax];
    int bytes[kReadbackMax]; // multiples of 4
    int dst[kReadbackMax];   // index of the first 8-byte host word
    int n;
    bool overflow;
    void add(const void *p, int nbytes, int word)
    {
        if (n >= kReadbackMax)
        {
            overflow = true;
            return;
        }
        src[n] = p;
        bytes[n] = nbytes;
        dst[n] = word;
        ++n;
    }
};

// Writes the readback words into mapped host memory from a kernel: a
// cudaMemcpyAsync would queue on a copy engine, where it waits behind any
// large copy another stream has queued (such as the previous conversion's
// outputs going to the host), and the host would wait with it.
__global__ void readback(Readback r, unsigned long long *host)
{
    const int i = threadIdx.x;
    if (i >= r.n)
        return;
    const uint32_t *s = (const uint32_t *)r.src[i];
    volatile uint32_t *d = (volatile uint32_t *)(host + r.dst[i]);
    for (int k = 0; k < r.bytes[i] / 4; ++k)
        d[k] = s[k];
    __threadfence_system();
}

uint32_t cap_u32(const Buf &b, size_t elem)
{
    const size_t n = b.cap / elem;
    return (uint32_t)(n < 0xffffffffull ? n : 0xffffffffull);
}

int status_to_error(ovx_fdg_context *ctx, uint32_t st)
{
    if (st & ST_BAD_INDEX)
        return fail(ctx, OVX_FDG_BAD_FACE_INDEX, "face index out of range [0, num_vertices)");
    if (st & ST_LIST_OVERFLOW)
        return fail(ctx, OVX_FDG_INTERNAL, "work list overflow");
    if (st & ST_REPLAY)
        return fail(ctx, OVX_FDG_INTERNAL, "record replay mismatch");
    if (st & ST_WALK_GUARD)
        return fail(ctx, OVX_FDG_INTERNAL, "boundary walk exceeded its step bound (non-finite vertex?)");
    return OVX_FDG_OK;
}

GenArgs make_gen(ovx_fdg_context *ctx)
{
    GenArgs A{};
    A.tune = ctx->tune;
    A.m = make_mesh(ctx);
    A.segs = ctx->batch ? (const Mesh *)ctx->segs_d.p : nullptr;
    A.nseg = ctx->batch ? (int)ctx->segs.size() : 0;
    A.bits = (uint32_t *)ctx->bits.p;
    A.rcnt = (uint32_t *)ctx->rcnt.p;
    A.roff = (const unsigned long long *)ctx->roff.p;
    A.rec = (Rec *)ctx->rec.p;
    A.qtab = (float *)ctx->qtab.p;
    A.btab = (float *)ctx->btab.p;
    // staging: event records, then face records, in the arena
    A.estage = ctx->estage_n ? (uint4 *)ctx->arena.p : nullptr;
    A.estage_cap = (uint32_t)ctx->estage_n;
    A.fstage = ctx->fstage_n ? (uint4 *)ctx->arena.p + ctx->estage_n : nullptr;
    A.fstage_cap = (uint32_t)ctx->fstage_n;
    A.counters = (uint32_t *)ctx->counters.p;
    A.scan_large = (uint32_t *)ctx->scan_large.p;
    A.scan_units = (uint32_t *)ctx->scan_units.p;
    // a list holds as many entries as its unit list holds beyond the total
    A.scan_large_cap = std::min(cap_u32(ctx->scan_large, 4), cap_u32(ctx->scan_units, 4) - 1u);
    A.face_large = (uint32_t *)ctx->face_large.p;
    A.face_units = (uint32_t *)ctx->face_units.p;
    A.face_large_cap = std::min(cap_u32(ctx->face_large, 4), cap_u32(ctx->face_units, 4) - 1u);
    A.bkeys = (const unsigned long long *)ctx->bkeys.p;
    A.bkeys_cap = cap_u32(ctx->bkeys, 8);
    A.blong = (uint32_t *)ctx->blong.p;
    A.blong_cap = cap_u32(ctx->blong, 4);
    return A;
}

// The in-place scan of a unit list (unit_tile_sums, unit_tile_offsets,
// unit_tile_scan); the occupancy pass sized unit_tiles for both lists.
cudaError_t unit_scan(ovx_fdg_context *ctx, uint32_t *units, uint32_t cap, uint32_t *counters, int count_word, int total_word,
                      cudaStream_t st)
{
    const uint32_t ntiles = cap / kUnitTile + 1;
    if ((size_t)ntiles * 8 > ctx->unit_tiles.cap)
        return cudaErrorInvalidValue;
    unsigned long long *tiles = (unsigned long long *)ctx->unit_tiles.p;
    unit_tile_sums<<<ntiles, kUnitTile, 0, st>>>(units, cap, counters, count_word, tiles);
    unit_tile_offsets<<<1, 1024, 0, st>>>(tiles, ntiles, units, cap, counters, count_word, total_word);
    unit_tile_scan<<<ntiles, kUnitTile, 0, st>>>(units, cap, counters, count_word, tiles);
    ctx->launches += 3;
    return cudaSuccess; // launch errors stay pending for the caller's check
}

template <int M, typename IdxT, bool B>
void launch_events(ovx_fdg_context *ctx, const GenArgs &A, cudaStream_t st)
{
    if (M == FILL && ctx->event_staged)
    {
        // the count pass staged the records of every pair
        if (ctx->n_estaged > 0)
        {
            bucket_records<<<blocks_for((long long)ctx->n_estaged, kThreads), kThreads, 0, st>>>(
                A.estage, (uint32_t)ctx->n_estaged, A.rcnt, A.roff, A.rec, A.counters);
            ++ctx->launches;
        }
    }
    else if (ctx->nf > 0)
    {
        tri_events<M, IdxT, B><<<blocks_for(3 * ctx->nf, kEventThreads), kEventThreads, 0, st>>>(A);
        ++ctx->launches;
        if (M == COUNT)
        {
            unit_scan(ctx, A.scan_units, A.scan_large_cap, A.counters, C_SCAN_LARGE, C_LUNITS, st);
        }
        // the fill pass knows the units (32 a warp); the count pass does not yet
        const long long rows_grid = M == FILL ? std::min<long long>(ctx->sms * 8, blocks_for((long long)ctx->n_lunits, kEventThreads))
                                              : ctx->sms * 8;
        if (rows_grid > 0)
        {
            large_rows<M, IdxT, B><<<(unsigned)rows_grid, kEventThreads, 0, st>>>(A);
            ++ctx->launches;
        }
    }
}

template <int M, typename IdxT, bool B>
void launch_faces_boundary(ovx_fdg_context *ctx, const GenArgs &A, cudaStream_t st)
{
    if (ctx->fw > 0.0f && ctx->nf > 0)
    {
        if (M == FILL && ctx->face_staged)
        {
            if (ctx->n_fstaged > 0)
            {
                place_records<<<blocks_for((long long)ctx->n_fstaged, kThreads), kThreads, 0, st>>>(
                    A.fstage, (uint32_t)ctx->n_fstaged, A.roff, A.rec, A.counters);
                ++ctx->launches;
            }
            // the boundary records follow the face records: the bucket cursors
            // as the count pass left them after the faces (a fill that runs
            // beside the event buckets uses that snapshot as its cursor)
            if (A.rcnt != (uint32_t *)ctx->face_end.p)
            {
                copy_words<<<blocks_for(ctx->g.nbricks + 1, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->face_end.p,
                                                                                        A.rcnt, ctx->g.nbricks + 1);
                ++ctx->launches;
            }
        }
        else
        {
            face_records<M, IdxT, B><<<blocks_for(ctx->nf, kFaceThreads), kFaceThreads, 0, st>>>(A);
            ++ctx->launches;
        }
        if (!(M == FILL && ctx->face_staged))
        {
            if (M == COUNT)
            {
                unit_scan(ctx, A.face_units, A.face_large_cap, A.counters, C_FACE_LARGE, C_FUNITS, st);
            }
            // one resident wave: the kernel loops over the units, and a second,
            // partial wave of CTAs only lengthens the tail
            static int per_sm = 0;
            if (per_sm < 1)
            {
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, large_faces<M, IdxT, B>, kFaceThreads, 0) != cudaSuccess ||
                    per_sm < 1)
                {
                    cudaGetLastError();
                    per_sm = 4;
                }
            }
            const long long wave = (long long)ctx->sms * per_sm;
            const long long faces_grid =
                M == FILL ? std::min<long long>(wave, blocks_for((long long)ctx->n_funits, kFaceThreads)) : wave;
            if (faces_grid > 0)
            {
                large_faces<M, IdxT, B><<<(unsigned)faces_grid, kFaceThreads, 0, st>>>(A);
                ++ctx->launches;
            }
        }
        if (M == COUNT && A.fstage)
        {
            // record counts after the scanline and face records, for the fill pass
            copy_words<<<blocks_for(ctx->g.nbricks + 1, kThreads), kThreads, 0, st>>>(A.rcnt, (uint32_t *)ctx->face_end.p,
                                                                                    ctx->g.nbricks + 1);
            ++ctx->launches;
        }
    }
    if (ctx->bw > 0.0f && ctx->nf > 0)
    {
        // at most 3F boundary edges; the fill pass knows the counts
        const long long nb_edges = M == FILL ? ctx->n_boundary : 3 * ctx->nf;
        const long long rec_grid = std::min<long long>(ctx->sms * 8, blocks_for(nb_edges, kThreads));
        if (rec_grid > 0)
        {
            boundary_records<M, B><<<(unsigned)rec_grid, kThreads, 0, st>>>(A);
            ++ctx->launches;
        }
        const long long nb_long = M == FILL ? (long long)ctx->n_blong : 3 * ctx->nf;
        const long long long_grid = std::min<long long>(ctx->sms * 4, blocks_for(nb_long, kThreads / 32));
        if (long_grid > 0)
        {
            boundary_long<M, B><<<(unsigned)long_grid, kThreads, 0, st>>>(A);
            ++ctx->launches;
        }
    }
}

// The record generators for the conversion in progress: batched, or a single
// mesh with int32 or int64 face indices.
template <int M>
void launch_events_any(ovx_fdg_context *ctx, const GenArgs &A, cudaStream_t st)
{
    if (ctx->batch)
        launch_events<M, int, true>(ctx, A, st);
    else if (ctx->fbytes == 8)
        launch_events<M, long long, false>(ctx, A, st);
    else
        launch_events<M, int, false>(ctx, A, st);
}

template <int M>
void launch_faces_boundary_any(ovx_fdg_context *ctx, const GenArgs &A, cudaStream_t st)
{
    if (ctx->batch)
        launch_faces_boundary<M, int, true>(ctx, A, st);
    else if (ctx->fbytes == 8)
        launch_faces_boundary<M, long long, false>(ctx, A, st);
    else
        launch_faces_boundary<M, int, false>(ctx, A, st);
}

// Occupancy stage shared by the full conversion and intersect_occ; ends with
// the one host synchronisation of a conversion.
int occupancy_pass(ovx_fdg_context *ctx, cudaStream_t st, bool full, int64_t *num_voxels, bool *retry)
{
    *retry = false;
    const Grid &g = ctx->g;
    const long long nf = ctx->nf, nb = g.nbricks;
    const bool boundary = full && ctx->bw > 0.0f;
    OVX_CUDA(ensure(st, ctx, ctx->bits, (size_t)nb * kWordsPerBrick * 4));
    OVX_CUDA(ensure(st, ctx, ctx->bcount, (size_t)(nb + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->bbase, (size_t)(nb + 1) * 8));
    OVX_CUDA(ensure(st, ctx, ctx->aflag, (size_t)(nb + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->aslot, (size_t)(nb + 1) * 8));
    OVX_CUDA(ensure(st, ctx, ctx->active, (size_t)(nb + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->counters, C_WORDS * 4));
    // work lists: the most entries seen, else a guess, never above the worst case
    auto list_room = [&](unsigned long long worst, unsigned long long want) {
        return std::min(worst, std::max(want, worst / 16 + ctx->list_guess));
    };
    const unsigned long long n_scan = list_room(3ull * nf, ctx->want_scan), n_face = list_room((unsigned long long)nf, ctx->want_face);
    OVX_CUDA(ensure(st, ctx, ctx->scan_large, (size_t)(n_scan + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->scan_units, (size_t)(n_scan + 2) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->face_large, (size_t)(n_face + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->face_units, (size_t)(n_face + 2) * 4));
    {
        // tile sums of the unit-list scans, for the lists as allocated
        const size_t tiles = std::max(cap_u32(ctx->scan_large, 4), cap_u32(ctx->face_large, 4)) / kUnitTile + 2;
        OVX_CUDA(ensure(st, ctx, ctx->unit_tiles, tiles * 8));
    }
    OVX_CUDA(ensure(st, ctx, ctx->rcnt, (size_t)(nb + 1) * 4));
    OVX_CUDA(ensure(st, ctx, ctx->roff, (size_t)(nb + 1) * 8));
    if (full)
        OVX_CUDA(ensure(st, ctx, ctx->qtab, (size_t)(nf + 1) * 48));
    ctx->estage_n = ctx->fstage_n = 0;
    if (full)
    {
        // staging room for the event records and then the face records, one
        // arena: for each, the most seen so far, else a guess
        const unsigned long long guess = std::min(24ull * (unsigned long long)nf, 4ull * (unsigned long long)nf + (16ull << 20));
        ctx->estage_n = std::min(std::max(ctx->estage_want, guess), 0xffffffffull);
        if (ctx->fw > 0.0f)
        {
            ctx->fstage_n = std::min(std::max(ctx->fstage_want, guess), 0xffffffffull);
            OVX_CUDA(ensure(st, ctx, ctx->face_end, (size_t)(nb + 1) * 4));
        }
        OVX_CUDA(ensure(st, ctx, ctx->arena, (size_t)(ctx->estage_n + ctx->fstage_n) * sizeof(uint4)));
    }
    if (boundary)
    {
        OVX_CUDA(ensure(st, ctx, ctx->vcnt, (size_t)(ctx->nv + 1) * 4));
        OVX_CUDA(ensure(st, ctx, ctx->voff, (size_t)(ctx->nv + 1) * 8));
        OVX_CUDA(ensure(st, ctx, ctx->emax, (size_t)(3 * nf + 1) * 4));
        OVX_CUDA(ensure(st, ctx, ctx->bkeys, (size_t)(list_room(3ull * nf, ctx->want_bkeys) + 1) * 8));
        OVX_CUDA(ensure(st, ctx, ctx->blong, (size_t)(list_room(3ull * nf, ctx->want_blong) + 1) * 4));
        OVX_CUDA(ensure(st, ctx, ctx->boff, (size_t)(ctx->nv + 1) * 8));
    }
    OVX_CUDA(cudaMemsetAsync(ctx->bits.p, 0, (size_t)nb * kWordsPerBrick * 4, st));
    OVX_CUDA(cudaMemsetAsync(ctx->counters.p, 0, C_WORDS * 4, st));
    OVX_CUDA(cudaMemsetAsync(ctx->rcnt.p, 0, (size_t)(nb + 1) * 4, st));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->bcount.p + nb, 0, 4, st));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->aflag.p + nb, 0, 4, st));

    if (boundary && nf > 0)
    {
        // undirected edges and the boundary list (edges used once), on the side
        // stream: they need only the mesh, so they run beside the scanline pass
        OVX_CUDA(side_stream(ctx));
        cudaStream_t es = ctx->side;
        OVX_CUDA(cudaEventRecord(ctx->fork_ev, st));
        OVX_CUDA(cudaStreamWaitEvent(es, ctx->fork_ev, 0));
        OVX_CUDA(cudaMemsetAsync(ctx->vcnt.p, 0, (size_t)(ctx->nv + 1) * 4, es));
        uint32_t *vcnt = (uint32_t *)ctx->vcnt.p;
        unsigned long long *voff = (unsigned long long *)ctx->voff.p;
        if (ctx->batch)
            edge_count_batch<<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const Mesh *)ctx->segs_d.p, (int)ctx->segs.size(), nf,
                                                                           vcnt);
        else if (ctx->fbytes == 8)
            edge_count<long long><<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const long long *)ctx->faces, nf, ctx->nv, vcnt);
        else
            edge_count<int><<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const int *)ctx->faces, nf, ctx->nv, vcnt);
        OVX_CUDA(cudaGetLastError());
        OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)vcnt, voff, ctx->nv + 1, es, &ctx->cub_tmp_side));
        if (ctx->batch)
            edge_fill_batch<<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const Mesh *)ctx->segs_d.p, (int)ctx->segs.size(), nf,
                                                                          voff, vcnt, (uint32_t *)ctx->emax.p);
        else if (ctx->fbytes == 8)
            edge_fill<long long><<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const long long *)ctx->faces, nf, ctx->nv, voff, vcnt,
                                                                               (uint32_t *)ctx->emax.p);
        else
            edge_fill<int><<<blocks_for(nf, kThreads), kThreads, 0, es>>>((const int *)ctx->faces, nf, ctx->nv, voff, vcnt,
                                                                         (uint32_t *)ctx->emax.p);
        OVX_CUDA(cudaGetLastError());
        // edge_fill left vcnt all zero: reuse it for the per-vertex boundary counts
        edge_sort_count<<<blocks_for(ctx->nv, kThreads), kThreads, 0, es>>>(voff, (uint32_t *)ctx->emax.p, ctx->nv, vcnt);
        OVX_CUDA(cudaGetLastError());
        unsigned long long *boff = (unsigned long long *)ctx->boff.p;
        OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)vcnt, boff, ctx->nv + 1, es, &ctx->cub_tmp_side));
        edge_emit<<<blocks_for(ctx->nv, kThreads), kThreads, 0, es>>>(voff, (const uint32_t *)ctx->emax.p, ctx->nv, boff,
                                                                     (unsigned long long *)ctx->bkeys.p,
                                                                     ctx->bkeys.cap / 8, (uint32_t *)ctx->counters.p);
        // boundary edge count -> counters[C_BOUNDARY] (low word of the u64 total; at most 3F < 2^32), by a
        // kernel rather than a copy, which could queue behind another stream's large copy
        copy_word<<<1, 1, 0, es>>>((const uint32_t *)(boff + ctx->nv), (uint32_t *)ctx->counters.p + C_BOUNDARY);
        ctx->launches += 5;
        OVX_CUDA(cudaGetLastError());
        OVX_CUDA(cudaEventRecord(ctx->join_ev, es));
    }
    stage(ctx, EV_BEGIN, st);
    GenArgs A = make_gen(ctx);
    if (!full)
    {
        A.qtab = nullptr;
        A.estage = nullptr; // occupancy only: no records
        A.estage_cap = 0;
    }
    launch_events_any<COUNT>(ctx, A, st);
    OVX_CUDA(cudaGetLastError());
    stage(ctx, EV_EVENTS_COUNT, st);

    brick_count<<<blocks_for(nb, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->bits.p, nb, (uint32_t *)ctx->bcount.p,
                                                               (uint32_t *)ctx->aflag.p);
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->bcount.p, (unsigned long long *)ctx->bbase.p, nb + 1, st));
    OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->aflag.p, (unsigned long long *)ctx->aslot.p, nb + 1, st));
    brick_slots<<<blocks_for(nb, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->aflag.p, (const unsigned long long *)ctx->aslot.p,
                                                               nb, (uint32_t *)ctx->active.p);
    ctx->launches += 2;
    if (ctx->batch)
    {
        const int ns = (int)ctx->segs.size();
        seg_rows<<<blocks_for(ns + 1, kThreads), kThreads, 0, st>>>((Mesh *)ctx->segs_d.p, ns,
                                                                   (const unsigned long long *)ctx->bbase.p, nb, ctx->seg_rows_dev);
        ++ctx->launches;
    }
    OVX_CUDA(cudaGetLastError());
    stage(ctx, EV_COMPACT, st);

    if (boundary && nf > 0)
        OVX_CUDA(cudaStreamWaitEvent(st, ctx->join_ev, 0)); // the boundary edges, from the side stream
    stage(ctx, EV_EDGES, st);

    if (full)
    {
        A = make_gen(ctx);
        launch_faces_boundary_any<COUNT>(ctx, A, st);
        OVX_CUDA(cudaGetLastError());
        OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->rcnt.p, (unsigned long long *)ctx->roff.p, nb + 1, st));
    }
    stage(ctx, EV_RECORD_COUNT, st);

    {
        Readback r{};
        r.add((unsigned long long *)ctx->bbase.p + nb, 8, 0);
        r.add((unsigned long long *)ctx->aslot.p + nb, 8, 1);
        if (full)
            r.add((unsigned long long *)ctx->roff.p + nb, 8, 2);
        r.add(ctx->counters.p, C_WORDS * 4, kHostCounters);
        if (r.overflow)
            return fail(ctx, OVX_FDG_INTERNAL, "readback list overflow");
        readback<<<1, 32, 0, st>>>(r, ctx->host_dev);
        ++ctx->launches;
    }
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(cudaStreamSynchronize(st));
    if (ctx->grew)
    {
        // the blocks freed by growth (this conversion's and the last one's) are
        // no longer in use: give them back instead of holding them
        ctx->grew = false;
        if (cudaMemPoolTrimTo(ctx->pool, 0) != cudaSuccess)
            cudaGetLastError();
    }
    const uint32_t *hc = (const uint32_t *)&ctx->host[kHostCounters];
    if (hc[C_STATUS] == (uint32_t)ST_LIST_OVERFLOW)
    {
        // a work list was too small: the counters hold the exact entry counts
        const GenArgs caps = make_gen(ctx); // the capacities the kernels used
        const bool over = hc[C_SCAN_LARGE] > caps.scan_large_cap || hc[C_FACE_LARGE] > caps.face_large_cap ||
                          (boundary && (hc[C_BLONG] > caps.blong_cap || hc[C_BOUNDARY] > caps.bkeys_cap));
        if (over)
        {
            ctx->want_scan = std::max(ctx->want_scan, (unsigned long long)hc[C_SCAN_LARGE]);
            ctx->want_face = std::max(ctx->want_face, (unsigned long long)hc[C_FACE_LARGE]);
            if (boundary)
            {
                ctx->want_blong = std::max(ctx->want_blong, (unsigned long long)hc[C_BLONG]);
                ctx->want_bkeys = std::max(ctx->want_bkeys, (unsigned long long)hc[C_BOUNDARY]);
            }
            *retry = true;
            return OVX_FDG_OK;
        }
    }
    const int rc = status_to_error(ctx, hc[C_STATUS]);
    if (rc != OVX_FDG_OK)
        return rc;
    const unsigned long long n = ctx->host[0];
    if (n >= (1ull << 31))
        return fail(ctx, OVX_FDG_CAPACITY, "more than 2^31-1 occupied voxels");
    ctx->n_vox = (long long)n;
    ctx->n_active = (long long)ctx->host[1];
    ctx->n_rec = full ? (long long)ctx->host[2] : 0;
    ctx->n_boundary = hc[C_BOUNDARY];
    ctx->n_lunits = hc[C_LUNITS];
    ctx->n_funits = hc[C_FUNITS];
    ctx->n_blong = hc[C_BLONG];
    ctx->n_estaged = full ? hc[C_ESTAGED] : 0u;
    ctx->event_staged = full && ctx->n_estaged <= ctx->estage_n;
    ctx->estage_want = std::max(ctx->estage_want, ctx->n_estaged);
    ctx->n_fstaged = full ? hc[C_FSTAGED] : 0u;
    ctx->face_staged = full && ctx->n_fstaged <= ctx->fstage_n;
    ctx->fstage_want = std::max(ctx->fstage_want, ctx->n_fstaged);
    // contribution entries: four per scanline event, one per face or boundary record
    ctx->n_events = full ? hc[C_EVENTS] : 0u;
    ctx->n_contrib = full ? 4ull * ctx->n_events + ((unsigned long long)ctx->n_rec - ctx->n_estaged) : 0ull;
    *num_voxels = (int64_t)n;
    return OVX_FDG_OK;
}

// The occupancy pass, run again with larger work lists when one overflowed.
// A pass counts every list's entries in full except the long boundary edges
// when the boundary list itself overflowed (only the edges that fitted were
// walked), so a second replay may be needed; each replay only grows a list.
int occupancy_stage(ovx_fdg_context *ctx, cudaStream_t st, bool full, int64_t *num_voxels)
{
    for (int attempt = 0;; ++attempt)
    {
        bool retry = false;
        const int rc = occupancy_pass(ctx, st, full, num_voxels, &retry);
        if (rc != OVX_FDG_OK || !retry)
            return rc;
        if (attempt >= 3)
            return fail(ctx, OVX_FDG_INTERNAL, "work list overflow");
    }
}

// The per-brick lists, the per-voxel sums and solves, and the constrained
// search of a conversion (single mesh or batch).
template <bool B, int P>
int launch_consume(ovx_fdg_context *ctx, const SolveArgs &SA, cudaStream_t st, long long n)
{
    if (ctx->n_active > 0)
    {
        brick_lists<B><<<(unsigned)ctx->n_active, kConsumeThreads, 0, st>>>(SA);
        ++ctx->launches;
    }
    stage(ctx, EV_CONSUME, st);
    voxel_accumulate<B, P><<<blocks_for(n, 128), 128, 0, st>>>(SA, n);
    // one CTA per long list, at most one per row
    voxel_accumulate_long<kLongMidMax, 128, false, B, P>
        <<<(unsigned)std::min<long long>(ctx->sms * 8, n), 128, long_smem<kLongMidMax>(), st>>>(SA);
    OVX_CUDA(cudaFuncSetAttribute(voxel_accumulate_long<kLongHugeMax, 256, true, B, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)long_smem<kLongHugeMax>()));
    voxel_accumulate_long<kLongHugeMax, 256, true, B, P>
        <<<(unsigned)std::min<long long>(ctx->sms * 2, n), 256, long_smem<kLongHugeMax>(), st>>>(SA);
    ctx->launches += 3;
    stage(ctx, EV_SOLVE, st);
    constrained_solve<B><<<(unsigned)std::min<long long>(ctx->sms * 8, blocks_for(n, 128)), 128, 0, st>>>(
        SA.clist, (const uint32_t *)ctx->counters.p, SA.clist_cap, ctx->g, SA.segs, SA.nseg, SA.dual);
    ++ctx->launches;
    OVX_CUDA(cudaGetLastError());
    return OVX_FDG_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int ovx_fdg_context_create(int device, ovx_fdg_context **out)
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
    ovx_fdg_context *ctx = new ovx_fdg_context();
    ctx->device = device;
    if (const char *lim = std::getenv("OVX_FDG_CLIST_LIMIT"))
        ctx->clist_limit = std::max(0ll, std::atoll(lim));
    if (const char *gs = std::getenv("OVX_FDG_LIST_GUESS"))
        ctx->list_guess = (unsigned long long)std::max(1ll, std::atoll(gs));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaHostAlloc((void **)&ctx->host, kHostWords * sizeof(unsigned long long), cudaHostAllocMapped);
    if (e == cudaSuccess)
        e = cudaHostGetDevicePointer((void **)&ctx->host_dev, ctx->host, 0);
    if (e == cudaSuccess)
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&ctx->pool, &props);
        if (e == cudaSuccess)
        {
            // freed blocks stay with the pool for the next growth instead of
            // going back to the driver at every synchronisation
            unsigned long long keep = ~0ull;
            e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        else
            ctx->pool = nullptr;
    }
    cudaSetDevice(prev);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        if (ctx->pool)
            cudaMemPoolDestroy(ctx->pool);
        if (ctx->host)
            cudaFreeHost(ctx->host);
        delete ctx;
        return OVX_FDG_OUT_OF_MEMORY;
    }
    *out = ctx;
    return OVX_FDG_OK;
}

void ovx_fdg_context_destroy(ovx_fdg_context *ctx)
{
    if (!ctx)
        return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    Buf *list[48];
    const int n = buffer_list(ctx, list);
    for (int i = 0; i < n; ++i)
        if (list[i]->p)
            cudaFree(list[i]->p); // waits for the device, then returns the block to the pool
    if (ctx->pool)
        cudaMemPoolDestroy(ctx->pool);
    if (ctx->host)
        cudaFreeHost(ctx->host);
    if (ctx->segs_pinned)
        cudaFreeHost(ctx->segs_pinned);
    if (ctx->seg_rows)
        cudaFreeHost(ctx->seg_rows);
    if (ctx->done)
        cudaEventDestroy(ctx->done);
    if (ctx->side)
        cudaStreamDestroy(ctx->side);
    if (ctx->fork_ev)
        cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev)
        cudaEventDestroy(ctx->join_ev);
    for (int i = 0; i < kStageEvents; ++i)
        if (ctx->ev[i])
            cudaEventDestroy(ctx->ev[i]);
    cudaSetDevice(prev);
    delete ctx;
}

int ovx_fdg_set_tuning(ovx_fdg_context *ctx, const ovx_fdg_tuning *t)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (!t)
    {
        ctx->tune = Tuning{kUnitCells, kWarpScanWork, kInlineFaceBricks, kDenseCandidates, kLongWalk};
        return OVX_FDG_OK;
    }
    if (t->unit_cells < 8 || t->unit_cells > 4096 || t->warp_scan_cells < 1 || t->warp_scan_cells > (1 << 20) ||
        t->inline_face_bricks < 1 || t->inline_face_bricks > 4096 || t->dense_candidates < 0 ||
        t->dense_candidates > kFaceWindow || t->long_walk < 1 || t->long_walk > (1 << 20))
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "tuning value out of range");
    ctx->tune = Tuning{t->unit_cells, t->warp_scan_cells, t->inline_face_bricks, t->dense_candidates, t->long_walk};
    return OVX_FDG_OK;
}

int ovx_fdg_get_tuning(const ovx_fdg_context *ctx, ovx_fdg_tuning *t)
{
    if (!ctx || !t)
        return OVX_FDG_INVALID_ARGUMENT;
    t->unit_cells = ctx->tune.unit_cells;
    t->warp_scan_cells = ctx->tune.scan_work;
    t->inline_face_bricks = ctx->tune.inline_face_bricks;
    t->dense_candidates = ctx->tune.dense_candidates;
    t->long_walk = ctx->tune.long_walk;
    return OVX_FDG_OK;
}

int ovx_fdg_set_precision(ovx_fdg_context *ctx, int precision, float route_tolerance)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (precision != OVX_FDG_PRECISION_EXACT && precision != OVX_FDG_PRECISION_COMPENSATED)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "unknown precision mode");
    if (!(route_tolerance >= 0.0f) || !(route_tolerance < 3.0e38f))
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "route tolerance must be finite and not negative");
    ctx->precision = precision;
    ctx->route_tol = route_tolerance;
    return OVX_FDG_OK;
}

int ovx_fdg_set_output_order(ovx_fdg_context *ctx, int order)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (order != OVX_FDG_ORDER_BRICK && order != OVX_FDG_ORDER_Z)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "unknown output order");
    ctx->order = order;
    return OVX_FDG_OK;
}

int ovx_fdg_pack(void *stream, const int32_t *voxel_indices, const float *dual_vertices, const uint8_t *intersected,
                 int64_t n, const float resolution[3], uint8_t *dual_u8, uint8_t *intersected_u8)
{
    if (n < 0 || !resolution || (n > 0 && (!voxel_indices || !dual_vertices || !intersected || !dual_u8 || !intersected_u8)))
        return OVX_FDG_INVALID_ARGUMENT;
    if (n == 0)
        return OVX_FDG_OK;
    fdg_pack_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(voxel_indices, dual_vertices, intersected, n, resolution[0],
                                                                          resolution[1], resolution[2], dual_u8, intersected_u8);
    return cudaGetLastError() == cudaSuccess ? OVX_FDG_OK : OVX_FDG_CUDA_ERROR;
}

int ovx_z_order_encode(void *stream, const int32_t *x, const int32_t *y, const int32_t *z, int64_t n, int32_t *codes)
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !codes)))
        return OVX_FDG_INVALID_ARGUMENT;
    if (n == 0)
        return OVX_FDG_OK;
    z_order_encode_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, y, z, n, codes);
    return cudaGetLastError() == cudaSuccess ? OVX_FDG_OK : OVX_FDG_CUDA_ERROR;
}

int ovx_z_order_decode(void *stream, const int32_t *codes, int64_t n, int32_t *x, int32_t *y, int32_t *z)
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !codes)))
        return OVX_FDG_INVALID_ARGUMENT;
    if (n == 0)
        return OVX_FDG_OK;
    z_order_decode_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(codes, n, x, y, z);
    return cudaGetLastError() == cudaSuccess ? OVX_FDG_OK : OVX_FDG_CUDA_ERROR;
}

int ovx_hilbert_encode(void *stream, const int32_t *x, const int32_t *y, const int32_t *z, int64_t n, int32_t *codes)
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !codes)))
        return OVX_FDG_INVALID_ARGUMENT;
    if (n == 0)
        return OVX_FDG_OK;
    hilbert_encode_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, y, z, n, codes);
    return cudaGetLastError() == cudaSuccess ? OVX_FDG_OK : OVX_FDG_CUDA_ERROR;
}

int ovx_hilbert_decode(void *stream, const int32_t *codes, int64_t n, int32_t *x, int32_t *y, int32_t *z)
{
    if (n < 0 || (n > 0 && (!x || !y || !z || !codes)))
        return OVX_FDG_INVALID_ARGUMENT;
    if (n == 0)
        return OVX_FDG_OK;
    hilbert_decode_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(codes, n, x, y, z);
    return cudaGetLastError() == cudaSuccess ? OVX_FDG_OK : OVX_FDG_CUDA_ERROR;
}

int ovx_fdg_set_profiling(ovx_fdg_context *ctx, int enable)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    if (enable)
        for (int i = 0; i < kStageEvents; ++i)
            if (!ctx->ev[i])
                OVX_CUDA(cudaEventCreate(&ctx->ev[i]));
    ctx->profiling = enable != 0;
    return OVX_FDG_OK;
}

int ovx_fdg_stage_times(ovx_fdg_context *ctx, float *ms, int capacity)
{
    if (!ctx || !ms)
        return -OVX_FDG_INVALID_ARGUMENT;
    if (!ctx->profiling)
        return 0;
    const int pairs[kStages][2] = {{EV_BEGIN, EV_EVENTS_COUNT}, {EV_EVENTS_COUNT, EV_COMPACT}, {EV_COMPACT, EV_EDGES},
                                   {EV_EDGES, EV_RECORD_COUNT}, {EV_FINISH, EV_EVENTS_FILL}, {EV_EVENTS_FILL, EV_RECORD_FILL},
                                   {EV_RECORD_FILL, EV_CONSUME}, {EV_CONSUME, EV_SOLVE}, {EV_SOLVE, EV_CONSTRAINED}};
    if (cudaEventSynchronize(ctx->ev[EV_CONSTRAINED]) != cudaSuccess)
    {
        cudaGetLastError();
        return -OVX_FDG_CUDA_ERROR;
    }
    int n = 0;
    for (int i = 0; i < kStages && i < capacity; ++i, ++n)
    {
        float t = -1.0f;
        if (cudaEventElapsedTime(&t, ctx->ev[pairs[i][0]], ctx->ev[pairs[i][1]]) != cudaSuccess)
        {
            cudaGetLastError();
            t = -1.0f;
        }
        ms[i] = t;
    }
    return n;
}

const char *ovx_fdg_stage_name(int i)
{
    return (i >= 0 && i < kStages) ? kStageNames[i] : "";
}

int64_t ovx_fdg_kernel_launches(const ovx_fdg_context *ctx)
{
    return ctx ? (int64_t)ctx->launches : 0;
}

int ovx_fdg_last_counts(const ovx_fdg_context *ctx, int64_t *out, int capacity)
{
    if (!ctx || (!out && capacity > 0) || capacity < 0)
        return -OVX_FDG_INVALID_ARGUMENT;
    const int64_t routed = (int64_t)((const uint32_t *)&ctx->host[kHostFinish])[C_ROUTED];
    const int64_t v[6] = {ctx->n_vox, ctx->n_active, ctx->n_rec, ctx->n_boundary, ctx->g.nbricks, routed};
    const int n = capacity < 6 ? capacity : 6;
    for (int i = 0; i < n; ++i)
        out[i] = v[i];
    return n;
}

const char *ovx_fdg_status_string(int status)
{
    switch (status)
    {
    case OVX_FDG_OK:
        return "ok";
    case OVX_FDG_INVALID_ARGUMENT:
        return "invalid argument";
    case OVX_FDG_BAD_FACE_INDEX:
        return "face index out of range";
    case OVX_FDG_CUDA_ERROR:
        return "CUDA error";
    case OVX_FDG_OUT_OF_MEMORY:
        return "out of device memory";
    case OVX_FDG_CAPACITY:
        return "input or result too large";
    case OVX_FDG_INTERNAL:
        return "internal bound exceeded";
    default:
        return "unknown status";
    }
}

const char *ovx_fdg_last_error(const ovx_fdg_context *ctx)
{
    return ctx ? ctx->err.c_str() : "no context";
}

int64_t ovx_fdg_workspace_bytes(const ovx_fdg_context *ctx)
{
    if (!ctx)
        return 0;
    Buf *list[48];
    const int n = buffer_list(const_cast<ovx_fdg_context *>(ctx), list);
    int64_t s = 0;
    for (int i = 0; i < n; ++i)
        s += (int64_t)list[i]->cap;
    // what the pool holds on the device, freed blocks it kept included
    unsigned long long reserved = 0;
    if (ctx->pool && cudaMemPoolGetAttribute(ctx->pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess)
        s = std::max(s, (int64_t)reserved);
    else
        cudaGetLastError();
    return s;
}

int ovx_fdg_begin(ovx_fdg_context *ctx, void *stream, const float *vertices, int64_t num_vertices, const void *faces,
                  int32_t face_index_bytes, int64_t num_faces, const float *origin, const ovx_fdg_grid *grid,
                  float face_weight, float boundary_weight, float regularization_weight, int64_t *num_voxels)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    ctx->phase = 0;
    ctx->err.clear();
    if (!num_voxels)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "num_voxels is NULL");
    *num_voxels = 0;
    if (num_vertices < 0 || num_faces < 0)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "negative size");
    if (num_faces > 0 && num_vertices == 0)
        return fail(ctx, OVX_FDG_BAD_FACE_INDEX, "faces reference vertices but there are none");
    if ((num_vertices > 0 && !vertices) || (num_faces > 0 && !faces))
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL vertices or faces");
    if (face_index_bytes != 4 && face_index_bytes != 8)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "face_index_bytes must be 4 or 8");
    if (num_faces > kMaxTriangles || num_vertices >= (1ll << 31) - 1)
        return fail(ctx, OVX_FDG_CAPACITY, "more than 2^28-1 faces or 2^31-2 vertices");
    Grid g{};
    int rc = check_grid(ctx, grid, g);
    if (rc != OVX_FDG_OK)
        return rc;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    ctx->batch = false;
    ctx->g = g;
    ctx->verts = vertices;
    ctx->nv = num_vertices;
    ctx->faces = faces;
    ctx->fbytes = face_index_bytes;
    ctx->nf = num_faces;
    for (int a = 0; a < 3; ++a)
        ctx->origin[a] = origin ? origin[a] : 0.0f;
    ctx->fw = face_weight;
    ctx->bw = boundary_weight;
    ctx->rw = regularization_weight;
    OVX_CUDA(wait_previous(ctx, (cudaStream_t)stream));
    rc = occupancy_stage(ctx, (cudaStream_t)stream, true, num_voxels);
    if (rc != OVX_FDG_OK)
        return rc;
    ctx->phase = 1;
    return OVX_FDG_OK;
}

int ovx_fdg_begin_batch(ovx_fdg_context *ctx, void *stream, const ovx_fdg_mesh *meshes, int32_t num_meshes, float face_weight,
                        float boundary_weight, float regularization_weight, int64_t *num_voxels, int64_t *total_voxels)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    ctx->phase = 0;
    ctx->err.clear();
    if (!total_voxels || !num_voxels || !meshes || num_meshes < 1)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "batch: NULL argument or no meshes");
    *total_voxels = 0;
    std::vector<Mesh> segs((size_t)num_meshes);
    long long tri = 0, brick = 0, vert = 0;
    for (int i = 0; i < num_meshes; ++i)
    {
        const ovx_fdg_mesh &m = meshes[i];
        num_voxels[i] = 0;
        const std::string which = "batch mesh " + std::to_string(i) + ": ";
        if (m.num_vertices < 0 || m.num_faces < 0)
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, (which + "negative size").c_str());
        if (m.num_faces > 0 && m.num_vertices == 0)
            return fail(ctx, OVX_FDG_BAD_FACE_INDEX, (which + "faces reference vertices but there are none").c_str());
        if ((m.num_vertices > 0 && !m.vertices) || (m.num_faces > 0 && !m.faces))
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, (which + "NULL vertices or faces").c_str());
        if (m.face_index_bytes != 4 && m.face_index_bytes != 8)
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, (which + "face_index_bytes must be 4 or 8").c_str());
        Grid g{};
        const int rc = check_grid(ctx, &m.grid, g);
        if (rc != OVX_FDG_OK)
        {
            ctx->err = which + ctx->err;
            return rc;
        }
        Mesh &M = segs[(size_t)i];
        M.g = g;
        M.verts = m.vertices;
        M.nv = m.num_vertices;
        M.faces = m.faces;
        M.nf = m.num_faces;
        M.ox = m.origin[0];
        M.oy = m.origin[1];
        M.oz = m.origin[2];
        M.fbytes = m.face_index_bytes;
        M.tri0 = tri;
        M.brick0 = brick;
        M.vert0 = vert;
        M.row0 = 0;
        tri += m.num_faces;
        brick += g.nbricks;
        vert += m.num_vertices;
    }
    if (tri > kMaxTriangles || vert >= (1ll << 31) - 1)
        return fail(ctx, OVX_FDG_CAPACITY, "batch: more than 2^28-1 faces or 2^31-2 vertices in all");
    if (brick >= (1ll << 31) || brick * kWordsPerBrick * 4ll > (64ll << 30))
        return fail(ctx, OVX_FDG_CAPACITY, "batch: grids too large for the dense brick bitmap (64 GiB limit)");
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    cudaStream_t st = (cudaStream_t)stream;
    OVX_CUDA(wait_previous(ctx, st));
    if (num_meshes > ctx->seg_cap)
    {
        // the previous batch's table upload and row readback are complete: its begin synchronised
        if (ctx->segs_pinned)
            cudaFreeHost(ctx->segs_pinned);
        if (ctx->seg_rows)
            cudaFreeHost(ctx->seg_rows);
        ctx->segs_pinned = nullptr;
        ctx->seg_rows = nullptr;
        ctx->seg_cap = 0;
        OVX_CUDA(cudaHostAlloc((void **)&ctx->segs_pinned, (size_t)num_meshes * sizeof(Mesh), cudaHostAllocMapped));
        OVX_CUDA(cudaHostAlloc((void **)&ctx->seg_rows, (size_t)(num_meshes + 1) * 8, cudaHostAllocMapped));
        OVX_CUDA(cudaHostGetDevicePointer((void **)&ctx->seg_rows_dev, ctx->seg_rows, 0));
        ctx->seg_cap = num_meshes;
    }
    std::memcpy(ctx->segs_pinned, segs.data(), (size_t)num_meshes * sizeof(Mesh));
    Mesh *segs_map = nullptr;
    OVX_CUDA(cudaHostGetDevicePointer((void **)&segs_map, ctx->segs_pinned, 0));
    static_assert(sizeof(Mesh) % 4 == 0, "the mesh table is copied in 32-bit words");
    OVX_CUDA(ensure(st, ctx, ctx->segs_d, (size_t)num_meshes * sizeof(Mesh)));
    const long long words = (long long)num_meshes * (long long)(sizeof(Mesh) / 4);
    load_segs<<<(unsigned)std::min<long long>(ctx->sms, blocks_for(words, kThreads)), kThreads, 0, st>>>(
        (const uint32_t *)segs_map, (uint32_t *)ctx->segs_d.p, words);
    ++ctx->launches;
    OVX_CUDA(cudaGetLastError());
    ctx->segs = std::move(segs);
    ctx->batch = true;
    ctx->g = Grid{};
    ctx->g.nbricks = brick;
    ctx->verts = nullptr;
    ctx->nv = vert;
    ctx->faces = nullptr;
    ctx->fbytes = 4;
    ctx->nf = tri;
    ctx->origin[0] = ctx->origin[1] = ctx->origin[2] = 0.0f;
    ctx->fw = face_weight;
    ctx->bw = boundary_weight;
    ctx->rw = regularization_weight;
    const int rc = occupancy_stage(ctx, st, true, total_voxels);
    if (rc != OVX_FDG_OK)
        return rc;
    for (int i = 0; i < num_meshes; ++i)
        num_voxels[i] = (int64_t)(ctx->seg_rows[i + 1] - ctx->seg_rows[i]);
    ctx->phase = 1;
    return OVX_FDG_OK;
}

int ovx_fdg_finish_batch(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices, float *dual_vertices, uint8_t *intersected)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (!ctx->batch || ctx->phase != 1)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "ovx_fdg_finish_batch without a successful ovx_fdg_begin_batch");
    return ovx_fdg_finish(ctx, stream, voxel_indices, dual_vertices, intersected);
}

int ovx_fdg_finish(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices, float *dual_vertices, uint8_t *intersected)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (ctx->phase != 1)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "ovx_fdg_finish without a successful ovx_fdg_begin");
    ctx->phase = 0;
    ctx->finished = 0;
    const long long n = ctx->n_vox;
    if (n == 0)
        return OVX_FDG_OK;
    if (!voxel_indices || !dual_vertices || !intersected)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL output buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    const long long nb = ctx->g.nbricks;
    // the record buffer holds the constrained-search list once the lists are built
    OVX_CUDA(ensure(st, ctx, ctx->rec, std::max((size_t)ctx->n_rec * sizeof(Rec), (size_t)64 * 1024)));
    OVX_CUDA(ensure(st, ctx, ctx->btab, (size_t)(ctx->n_boundary + 1) * 48));
    OVX_CUDA(ensure(st, ctx, ctx->vlist, (size_t)n * 8));
    OVX_CUDA(ensure(st, ctx, ctx->longv, (size_t)(n + 1) * 4));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->counters.p + C_LONG, 0, 4, st));
    OVX_CUDA(cudaMemsetAsync(ctx->rcnt.p, 0, (size_t)(nb + 1) * 4, st));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->counters.p + C_CONSTRAINED, 0, 4, st));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->counters.p + C_ROUTED, 0, 4, st));

    stage(ctx, EV_FINISH, st);
    GenArgs A = make_gen(ctx);
    A.qtab = nullptr;
    if (ctx->event_staged && ctx->face_staged && ctx->fw > 0.0f && ctx->bw > 0.0f && ctx->nf > 0 && ctx->side)
    {
        // every record was staged: the event buckets (cursor rcnt), the face
        // records (at their staged ranks) and the boundary records (cursor:
        // the per-brick counts after the faces, face_end) write disjoint
        // places, so the face and boundary fills run on the side stream
        // beside the event buckets
        OVX_CUDA(cudaEventRecord(ctx->fork_ev, st));
        OVX_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
        GenArgs Af = A;
        Af.rcnt = (uint32_t *)ctx->face_end.p;
        launch_faces_boundary_any<FILL>(ctx, Af, ctx->side);
        OVX_CUDA(cudaEventRecord(ctx->join_ev, ctx->side));
        launch_events_any<FILL>(ctx, A, st);
        stage(ctx, EV_EVENTS_FILL, st);
        OVX_CUDA(cudaStreamWaitEvent(st, ctx->join_ev, 0));
    }
    else
    {
        launch_events_any<FILL>(ctx, A, st);
        stage(ctx, EV_EVENTS_FILL, st);
        launch_faces_boundary_any<FILL>(ctx, A, st);
    }
    OVX_CUDA(cudaGetLastError());
    stage(ctx, EV_RECORD_FILL, st);
    // the staged records are in their buckets: the arena now takes the
    // contribution lists (a growth frees the old block behind the fills)
    OVX_CUDA(ensure(st, ctx, ctx->arena, (size_t)(ctx->n_contrib + 1) * sizeof(uint2)));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->counters.p + C_CONTRIB, 0, 8, st));

    SolveArgs SA{};
    SA.m = make_mesh(ctx);
    SA.segs = ctx->batch ? (const Mesh *)ctx->segs_d.p : nullptr;
    SA.nseg = ctx->batch ? (int)ctx->segs.size() : 0;
    SA.bw = ctx->bw;
    SA.rw = ctx->rw;
    SA.bits = (const uint32_t *)ctx->bits.p;
    SA.bbase = (const unsigned long long *)ctx->bbase.p;
    SA.zorder = ctx->order == 1;
    if (SA.zorder)
    {
        const int zr = zorder_row_bases(ctx, st);
        if (zr != OVX_FDG_OK)
            return zr;
        SA.bbase = (const unsigned long long *)ctx->zbase.p;
    }
    SA.active = (const uint32_t *)ctx->active.p;
    SA.roff = (const unsigned long long *)ctx->roff.p;
    SA.rec = (const Rec *)ctx->rec.p;
    SA.qtab = (const float *)ctx->qtab.p;
    SA.btab = (const float *)ctx->btab.p;
    SA.vox = voxel_indices;
    SA.dual = dual_vertices;
    SA.flags = intersected;
    SA.counters = (uint32_t *)ctx->counters.p;
    SA.clist = (float *)ctx->rec.p;
    SA.contrib = (uint2 *)ctx->arena.p;
    SA.contrib_cap = ctx->arena.cap / sizeof(uint2);
    SA.key_face = (uint32_t)(12 * ctx->nf);
    SA.key_boundary = (uint32_t)(13 * ctx->nf);
    SA.vlist = (unsigned long long *)ctx->vlist.p;
    SA.longv = (uint32_t *)ctx->longv.p;
    SA.longv_cap = (uint32_t)(n + 1);
    SA.clist_cap = (uint32_t)std::min<size_t>(ctx->rec.cap / 64, (size_t)n + 1);
    if (ctx->clist_limit >= 0)
        SA.clist_cap = (uint32_t)std::min<long long>(SA.clist_cap, ctx->clist_limit);
    SA.route_tol = ctx->route_tol;
    const int cr = ctx->batch ? (ctx->precision ? launch_consume<true, 1>(ctx, SA, st, n) : launch_consume<true, 0>(ctx, SA, st, n))
                              : (ctx->precision ? launch_consume<false, 1>(ctx, SA, st, n) : launch_consume<false, 0>(ctx, SA, st, n));
    if (cr != OVX_FDG_OK)
        return cr;
    stage(ctx, EV_CONSTRAINED, st);
    OVX_CUDA(cudaGetLastError());
    {
        Readback r{};
        r.add(ctx->counters.p, C_WORDS * 4, kHostFinish);
        if (r.overflow)
            return fail(ctx, OVX_FDG_INTERNAL, "readback list overflow");
        readback<<<1, 32, 0, st>>>(r, ctx->host_dev);
        ++ctx->launches;
    }
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(mark_done(ctx, st));
    ctx->finished = 1;
    return OVX_FDG_OK;
}

int ovx_fdg_sync_status(ovx_fdg_context *ctx, void *stream)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    OVX_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (!ctx->finished)
        return OVX_FDG_OK;
    ctx->finished = 0;
    return status_to_error(ctx, ((const uint32_t *)&ctx->host[kHostFinish])[C_STATUS]);
}

int ovx_fdg_occupancy_begin(ovx_fdg_context *ctx, void *stream, const float *triangles, int64_t num_triangles,
                            const ovx_fdg_grid *grid, int64_t *num_voxels)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    ctx->phase = 0;
    ctx->err.clear();
    if (!num_voxels)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "num_voxels is NULL");
    *num_voxels = 0;
    if (num_triangles < 0 || (num_triangles > 0 && !triangles))
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "bad triangles");
    if (num_triangles >= (1ll << 30))
        return fail(ctx, OVX_FDG_CAPACITY, "more than 2^30 triangles");
    Grid g{};
    int rc = check_grid(ctx, grid, g);
    if (rc != OVX_FDG_OK)
        return rc;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    ctx->batch = false;
    ctx->g = g;
    ctx->verts = triangles;
    ctx->nv = num_triangles * 3;
    ctx->faces = nullptr;
    ctx->fbytes = 4;
    ctx->nf = num_triangles;
    ctx->origin[0] = ctx->origin[1] = ctx->origin[2] = 0.0f;
    ctx->fw = 0.0f;
    ctx->bw = 0.0f;
    ctx->rw = 0.0f;
    OVX_CUDA(wait_previous(ctx, (cudaStream_t)stream));
    rc = occupancy_stage(ctx, (cudaStream_t)stream, false, num_voxels);
    if (rc != OVX_FDG_OK)
        return rc;
    ctx->phase = 2;
    return OVX_FDG_OK;
}

int ovx_fdg_occupancy_finish(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (ctx->phase != 2)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "ovx_fdg_occupancy_finish without a successful ovx_fdg_occupancy_begin");
    ctx->phase = 0;
    if (ctx->n_vox == 0)
        return OVX_FDG_OK;
    if (!voxel_indices)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL output buffer");
    cudaStream_t st = (cudaStream_t)stream;
    const DeviceScope scope(ctx->device);
    OVX_CUDA(scope.status);
    const unsigned long long *base = (const unsigned long long *)ctx->bbase.p;
    if (ctx->order == 1)
    {
        const int zr = zorder_row_bases(ctx, st);
        if (zr != OVX_FDG_OK)
            return zr;
        base = (const unsigned long long *)ctx->zbase.p;
    }
    brick_coords<<<(unsigned)ctx->n_active, 128, 0, st>>>((const uint32_t *)ctx->bits.p, base, (const uint32_t *)ctx->active.p,
                                                          ctx->g, ctx->order == 1, voxel_indices);
    ++ctx->launches;
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(mark_done(ctx, st));
    return OVX_FDG_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// allocation-free occupancy: host side
// ---------------------------------------------------------------------------
namespace
{
// Device address of the scratch array on the current device (the name itself
// is a host-side stand-in, not a device address).  Looked up on every call: the
// lookup is cheap, and a cached address would go stale if the caller reset the
// device (cudaDeviceReset reloads the module, which can place the array
// elsewhere).
cudaError_t noalloc_scratch(void **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
        return e;
    *out = p;
    return cudaSuccess;
}
} // namespace

extern "C" int ovx_fdg_occupancy_noalloc(void *stream, const float *triangles, int64_t num_triangles, const ovx_fdg_grid *grid,
                                         int32_t *voxel_indices, int64_t capacity, int64_t *num_voxels)
{
    if (!num_voxels || !grid || num_triangles < 0 || capacity < 0 || (num_triangles > 0 && !triangles) ||
        (capacity > 0 && !voxel_indices))
        return OVX_FDG_INVALID_ARGUMENT;
    *num_voxels = 0;
    if (num_triangles >= (1ll << 30))
        return OVX_FDG_CAPACITY;
    Grid g{};
    long long nb = 1;
    for (int a = 0; a < 3; ++a)
    {
        const float vs = grid->voxel_size[a];
        if (!(vs > 0.0f) || !(vs < 3.0e38f))
            return OVX_FDG_INVALID_ARGUMENT;
        const long long sz = (long long)grid->grid_max[a] - (long long)grid->grid_min[a];
        if (sz < 1 || sz > (1 << 20))
            return OVX_FDG_INVALID_ARGUMENT;
        g.vs[a] = vs;
        g.rv[a] = 1.0 / (double)vs;
        g.gmin[a] = grid->grid_min[a];
        g.gmax[a] = grid->grid_max[a];
        g.size[a] = (int)sz;
        g.nb[a] = (int)((sz + kBrick - 1) / kBrick);
        nb *= g.nb[a];
    }
    if (nb > kNoallocMaxBricks)
        return OVX_FDG_CAPACITY; // grid larger than the fixed scratch covers
    g.nbricks = nb;
    cudaStream_t st = (cudaStream_t)stream;
    // the call waits on the stream once (to read N), which a stream capture forbids
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess)
    {
        cudaGetLastError();
        return OVX_FDG_CUDA_ERROR;
    }
    if (cap != cudaStreamCaptureStatusNone)
        return OVX_FDG_INVALID_ARGUMENT;
    void *scratch = nullptr;
    if (noalloc_scratch(&scratch) != cudaSuccess)
    {
        cudaGetLastError();
        return OVX_FDG_CUDA_ERROR;
    }
    uint32_t *bits = (uint32_t *)scratch;
    uint32_t *base = (uint32_t *)((unsigned char *)scratch + kNoallocBitsBytes);
    noalloc_clear<<<256, 256, 0, st>>>(bits, nb * kWordsPerBrick);
    if (num_triangles > 0)
        noalloc_mark<<<blocks_for(3 * num_triangles, kThreads), kThreads, 0, st>>>(triangles, num_triangles, g, bits);
    noalloc_scan<<<1, 1024, 0, st>>>(bits, nb, base);
    uint32_t total = 0;
    if (cudaGetLastError() != cudaSuccess || cudaMemcpyAsync(&total, base + nb, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
    {
        cudaGetLastError();
        return OVX_FDG_CUDA_ERROR;
    }
    *num_voxels = (int64_t)total;
    if ((int64_t)total > capacity)
        return OVX_FDG_CAPACITY; // output buffer too small; *num_voxels says how many rows are needed
    if (total > 0)
        noalloc_emit<<<blocks_for(nb * kWordsPerBrick, kThreads), kThreads, 0, st>>>(bits, base, g, voxel_indices);
    if (cudaGetLastError() != cudaSuccess)
        return OVX_FDG_CUDA_ERROR;
    return OVX_FDG_OK;
}
