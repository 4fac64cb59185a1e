// fdg_kernels.cu -- B200 mesh -> flexible dual grid: kernels, host
// orchestration and the C ABI declared in include/ovx_fdg.h.
//
// Pipeline (one mesh; every stage is a plain SIMT kernel -- nothing here is a
// dense contraction, so there is no tensor-core work):
//
//  begin (occupancy)
//   tri_pass<MARK>        one thread per triangle: scanline events of the three
//                         projection axes (FP64, reference arithmetic) set bits in
//                         a dense brick-ordered occupancy bitmap; (triangle,axis)
//                         pairs with many events and triangles with a large face
//                         box go to two work lists.
//   large_scan<MARK>      one CTA per listed (triangle,axis), threads over
//                         (row, 8-column chunk) tiles.
//   brick_count + scan    popcount per 8^3 brick, exclusive scan -> N.
//   edge_* (boundary_weight>0)
//                         undirected edges bucketed by their smaller vertex
//                         (counting sort); edges used by one face -> boundary list.
//  finish (quadrics + solve)
//   brick_emit            voxel rows in brick order + per-word row bases.
//   *<COUNT>              replay events / face tests / boundary walks, count
//                         quadric contributions per voxel.
//   scan                  per-voxel segment offsets -> E.
//   *<FILL>               replay again, write (order key, payload) per contribution.
//   final_short/long      per voxel: sort its contributions by the reference's
//                         accumulation order, sum them sequentially in FP32 (the
//                         reference order, so the sums are bit-identical),
//                         regularise, solve, write dual vertex and flags.
//
// Order keys (64 bit, unique per voxel; ascending = reference CPU order,
// flexible_dual_grid.cpp:173-283, :298-414, :741-757):
//   intersection  (0<<62) | ((t*3 + axis)*4 + (1-dy)*2 + (1-dx))
//   face          (1<<62) | t
//   boundary      (2<<62) | (v_min<<31) | v_max
#include "ovx_fdg.h"
#include "fdg_device.cuh"

#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <cstring>
#include <string>

using namespace ovx;

namespace
{

enum Mode
{
    MARK = 0,
    COUNT = 1,
    FILL = 2
};

constexpr int kInlineScanWork = 256; // rows x column span of one (triangle, axis) done by the triangle's thread
constexpr int kInlineFaceVoxels = 64; // face-box voxels done by the triangle's thread
constexpr int kChunk = 8;            // columns per tile in the large path
constexpr int kShortSeg = 32;        // contributions per voxel sorted inside one thread
constexpr int kLongSmem = 2048;      // contributions per voxel sorted in shared memory by one CTA
constexpr int kThreads = 256;

// device counter words
enum
{
    C_SCAN_LARGE = 0,
    C_FACE_LARGE = 1,
    C_BOUNDARY = 2,
    C_LONG = 3,
    C_STATUS = 4,
    C_WORDS = 8
};
enum
{
    ST_BAD_INDEX = 1,
    ST_WALK_GUARD = 2,
    ST_LIST_OVERFLOW = 4,
    ST_REPLAY = 8
};

constexpr unsigned long long kStageFace = 1ull << 62;
constexpr unsigned long long kStageBoundary = 2ull << 62;

struct Pass
{
    Grid g;
    const float *verts;
    long long nv;
    const void *faces;
    long long nf;
    float ox, oy, oz;
    uint32_t *bits;
    const uint32_t *word_base;
    uint32_t *ecount;
    const unsigned long long *eseg;
    unsigned long long *ekey;
    uint32_t *epay;
    uint32_t *counters;
    uint32_t *scan_large;
    uint32_t scan_large_cap;
    uint32_t *face_large;
    uint32_t face_large_cap;
    const uint2 *blist;
    uint32_t blist_cap;
    int face_on;
};

// (u, v, w) are coordinates along (ax0, ax1, ax2) of projection axis ax2.
__device__ __forceinline__ void place(int ax2, int u, int v, int w, int &x, int &y, int &z)
{
    x = ax2 == 0 ? w : (ax2 == 1 ? v : u);
    y = ax2 == 0 ? u : (ax2 == 1 ? w : v);
    z = ax2 == 0 ? v : (ax2 == 1 ? u : w);
}

template <int M>
__device__ __forceinline__ void contribute(const Pass &P, long long w, uint32_t bit, unsigned long long key, uint32_t pay)
{
    const uint32_t m = 1u << bit;
    if (M == MARK)
    {
        if (!(P.bits[w] & m))
            atomicOr(&P.bits[w], m);
    }
    else
    {
        const uint32_t row = P.word_base[w] + __popc(P.bits[w] & (m - 1u));
        if (M == COUNT)
        {
            atomicAdd(&P.ecount[row], 1u);
        }
        else
        {
            const uint32_t left = atomicSub(&P.ecount[row], 1u);
            if (left == 0u)
            {
                // the replay produced more contributions than the count pass: never write out of the segment
                atomicOr(&P.counters[C_STATUS], (uint32_t)ST_REPLAY);
                return;
            }
            const unsigned long long pos = P.eseg[row] + (unsigned long long)(left - 1u);
            P.ekey[pos] = key;
            P.epay[pos] = pay;
        }
    }
}

template <int M>
struct EventSink
{
    const Pass &P;
    long long t;
    int ax2;
    __device__ __forceinline__ void operator()(int xi, int yi, int zi, float, float, double z) const
    {
        const uint32_t zb = __float_as_uint((float)z);
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
            {
                int x, y, zz;
                place(ax2, xi + dx, yi + dy, zi, x, y, zz);
                uint32_t bit;
                const long long w = voxel_word(P.g, x, y, zz, bit);
                const unsigned long long key = (unsigned long long)((t * 3 + ax2) * 4 + (1 - dy) * 2 + (1 - dx));
                contribute<M>(P, w, bit, key, zb);
            }
    }
};

__device__ __forceinline__ void face_box(const float v[3][3], const Grid &g, int bmin[3], int bmax[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        float mn = v[0][i], mx = v[0][i];
        mn = (v[1][i] < mn) ? v[1][i] : mn;
        mn = (v[2][i] < mn) ? v[2][i] : mn;
        mx = (mx < v[1][i]) ? v[1][i] : mx;
        mx = (mx < v[2][i]) ? v[2][i] : mx;
        const int l = trunc_f2i(mn / g.vs[i]);
        const int h = trunc_f2i(mx / g.vs[i] + 1.0f);
        bmin[i] = (l < g.gmin[i]) ? g.gmin[i] : l;
        bmax[i] = (g.gmax[i] < h) ? g.gmax[i] : h;
    }
}

template <typename IdxT>
__device__ __forceinline__ bool tri_load(const Pass &P, long long t, float v[3][3])
{
    long long idx[3];
    const float o[3] = {P.ox, P.oy, P.oz};
    return load_triangle<IdxT>(P.verts, P.nv, (const IdxT *)P.faces, t, o, v, idx);
}

// Face test of the active voxels of one brick inside the triangle's face box.
template <int M>
__device__ __forceinline__ void face_brick(const Pass &P, const FaceSetup &fs, long long t, int bx, int by, int bz)
{
    const Grid &g = P.g;
    const long long brick = (long long)bx + (long long)g.nb[0] * ((long long)by + (long long)g.nb[1] * (long long)bz);
    const int x0 = g.gmin[0] + bx * kBrick, y0 = g.gmin[1] + by * kBrick, z0 = g.gmin[2] + bz * kBrick;
    uint32_t xmask = 0;
#pragma unroll
    for (int lx = 0; lx < 8; ++lx)
        if (x0 + lx >= fs.bmin[0] && x0 + lx < fs.bmax[0])
            xmask |= 1u << lx;
    for (int w = 0; w < kWordsPerBrick; ++w)
    {
        const int z = z0 + (w >> 1);
        if (z < fs.bmin[2] || z >= fs.bmax[2])
            continue;
        uint32_t mask = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int y = y0 + (w & 1) * 4 + q;
            if (y >= fs.bmin[1] && y < fs.bmax[1])
                mask |= xmask << (q * 8);
        }
        uint32_t word = P.bits[brick * kWordsPerBrick + w] & mask;
        while (word)
        {
            const int b = __ffs(word) - 1;
            word &= word - 1u;
            const int x = x0 + (b & 7), y = y0 + (w & 1) * 4 + (b >> 3);
            if (face_test(fs, g, x, y, z))
                contribute<M>(P, brick * kWordsPerBrick + w, (uint32_t)b, kStageFace | (unsigned long long)t, 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// per-triangle pass
// ---------------------------------------------------------------------------
template <int M, typename IdxT>
__global__ void __launch_bounds__(kThreads) tri_pass(Pass P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.nf)
        return;
    float v[3][3];
    if (!tri_load<IdxT>(P, t, v))
    {
        if (M == MARK)
            atomicOr(&P.counters[C_STATUS], (uint32_t)ST_BAD_INDEX);
        return;
    }
#pragma unroll 1
    for (int ax2 = 0; ax2 < 3; ++ax2)
    {
        AxisScan s;
        axis_setup(v, ax2, P.g, s);
        const int rows = s.end - s.start;
        if (rows <= 0)
            continue;
        int clo, chi;
        axis_col_bounds(s, P.g, clo, chi);
        const long long work = (long long)rows * (long long)(chi - clo + 1);
        if (work > kInlineScanWork)
        {
            if (M == MARK)
            {
                const uint32_t slot = atomicAdd(&P.counters[C_SCAN_LARGE], 1u);
                if (slot < P.scan_large_cap)
                    P.scan_large[slot] = (uint32_t)(t * 3 + ax2);
                else
                    atomicOr(&P.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
            }
            continue;
        }
        EventSink<M> sink{P, t, ax2};
#pragma unroll 1
        for (int yi = s.start; yi < s.end; ++yi)
            scan_row(s, yi, INT_MIN, INT_MAX, P.g, sink);
    }
    if (!P.face_on)
        return;
    int bmin[3], bmax[3];
    face_box(v, P.g, bmin, bmax);
    const long long ex = bmax[0] - bmin[0], ey = bmax[1] - bmin[1], ez = bmax[2] - bmin[2];
    if (ex <= 0 || ey <= 0 || ez <= 0)
        return;
    if (ex * ey * ez > kInlineFaceVoxels)
    {
        if (M == MARK)
        {
            const uint32_t slot = atomicAdd(&P.counters[C_FACE_LARGE], 1u);
            if (slot < P.face_large_cap)
                P.face_large[slot] = (uint32_t)t;
            else
                atomicOr(&P.counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
        }
        return;
    }
    if (M == MARK)
        return;
    FaceSetup fs;
    face_setup(v, P.g, fs);
#pragma unroll 1
    for (int z = bmin[2]; z < bmax[2]; ++z)
#pragma unroll 1
        for (int y = bmin[1]; y < bmax[1]; ++y)
#pragma unroll 1
            for (int x = bmin[0]; x < bmax[0]; ++x)
            {
                uint32_t bit;
                const long long w = voxel_word(P.g, x, y, z, bit);
                if (!(P.bits[w] & (1u << bit)))
                    continue;
                if (face_test(fs, P.g, x, y, z))
                    contribute<M>(P, w, bit, kStageFace | (unsigned long long)t, 0u);
            }
}

// One CTA per listed (triangle, axis); threads over (row, column chunk) tiles.
template <int M, typename IdxT>
__global__ void __launch_bounds__(128) large_scan(Pass P)
{
    const uint32_t n = min(P.counters[C_SCAN_LARGE], P.scan_large_cap);
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
    {
        const uint32_t e = P.scan_large[i];
        const long long t = e / 3;
        const int ax2 = (int)(e % 3);
        float v[3][3];
        if (!tri_load<IdxT>(P, t, v))
            continue;
        AxisScan s;
        axis_setup(v, ax2, P.g, s);
        const int rows = s.end - s.start;
        int clo, chi;
        axis_col_bounds(s, P.g, clo, chi);
        const int nch = (chi - clo + 1 + kChunk - 1) / kChunk;
        const long long tiles = (long long)rows * nch;
        EventSink<M> sink{P, t, ax2};
        for (long long k = threadIdx.x; k < tiles; k += blockDim.x)
        {
            const int yi = s.start + (int)(k / nch);
            const int ch = (int)(k % nch);
            const int lo = ch == 0 ? INT_MIN : clo + ch * kChunk;
            const int hi = ch == nch - 1 ? INT_MAX : clo + (ch + 1) * kChunk;
            scan_row(s, yi, lo, hi, P.g, sink);
        }
    }
}

// One CTA per listed triangle; threads over the bricks of its face box.
template <int M, typename IdxT>
__global__ void __launch_bounds__(128) large_face(Pass P)
{
    const uint32_t n = min(P.counters[C_FACE_LARGE], P.face_large_cap);
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x)
    {
        const long long t = P.face_large[i];
        float v[3][3];
        if (!tri_load<IdxT>(P, t, v))
            continue;
        FaceSetup fs;
        face_setup(v, P.g, fs);
        const Grid &g = P.g;
        int b0[3], b1[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
        {
            b0[a] = (fs.bmin[a] - g.gmin[a]) >> 3;
            b1[a] = (fs.bmax[a] - 1 - g.gmin[a]) >> 3;
        }
        const long long nx = b1[0] - b0[0] + 1, ny = b1[1] - b0[1] + 1, nz = b1[2] - b0[2] + 1;
        const long long total = nx * ny * nz;
        for (long long k = threadIdx.x; k < total; k += blockDim.x)
        {
            const int bx = b0[0] + (int)(k % nx);
            const int by = b0[1] + (int)((k / nx) % ny);
            const int bz = b0[2] + (int)(k / (nx * ny));
            face_brick<M>(P, fs, t, bx, by, bz);
        }
    }
}

// Boundary walks, one thread per boundary edge.
template <int M>
__global__ void __launch_bounds__(kThreads) boundary_pass(Pass P)
{
    const uint32_t n = min(P.counters[C_BOUNDARY], P.blist_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const uint2 e = P.blist[i];
        float v0[3], v1[3];
        v0[0] = P.verts[(long long)e.x * 3 + 0] - P.ox;
        v0[1] = P.verts[(long long)e.x * 3 + 1] - P.oy;
        v0[2] = P.verts[(long long)e.x * 3 + 2] - P.oz;
        v1[0] = P.verts[(long long)e.y * 3 + 0] - P.ox;
        v1[1] = P.verts[(long long)e.y * 3 + 1] - P.oy;
        v1[2] = P.verts[(long long)e.y * 3 + 2] - P.oz;
        Dda d;
        if (!boundary_setup(v0, v1, P.g, d, nullptr))
            continue;
        const unsigned long long key = kStageBoundary | ((unsigned long long)e.x << 31) | (unsigned long long)e.y;
        for (;;)
        {
            if (in_grid(P.g, d.cur[0], d.cur[1], d.cur[2]))
            {
                uint32_t bit;
                const long long w = voxel_word(P.g, d.cur[0], d.cur[1], d.cur[2], bit);
                if (P.bits[w] & (1u << bit))
                    contribute<M>(P, w, bit, key, 0u);
            }
            if (!dda_step(d))
                break;
        }
        if (d.guard < 0)
            atomicOr(&P.counters[C_STATUS], (uint32_t)ST_WALK_GUARD);
    }
}

// ---------------------------------------------------------------------------
// occupancy compaction
// ---------------------------------------------------------------------------
__global__ void brick_count(const uint32_t *__restrict__ bits, long long nbricks, uint32_t *__restrict__ bcount)
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
}

// Row bases per occupancy word and voxel coordinates in brick order.
__global__ void brick_emit(const uint32_t *__restrict__ bits, const unsigned long long *__restrict__ bbase, Grid g,
                           uint32_t *__restrict__ word_base, int32_t *__restrict__ vox)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= g.nbricks)
        return;
    unsigned long long base = bbase[b];
    if (bbase[b + 1] == base)
        return;
    const int bx = (int)(b % g.nb[0]);
    const int by = (int)((b / g.nb[0]) % g.nb[1]);
    const int bz = (int)(b / ((long long)g.nb[0] * g.nb[1]));
    for (int w = 0; w < kWordsPerBrick; ++w)
    {
        uint32_t word = bits[b * kWordsPerBrick + w];
        if (word_base)
            word_base[b * kWordsPerBrick + w] = (uint32_t)base;
        while (word)
        {
            const int bit = __ffs(word) - 1;
            word &= word - 1u;
            const int li = w * 32 + bit;
            if (vox)
            {
                vox[base * 3 + 0] = g.gmin[0] + bx * kBrick + (li & 7);
                vox[base * 3 + 1] = g.gmin[1] + by * kBrick + ((li >> 3) & 7);
                vox[base * 3 + 2] = g.gmin[2] + bz * kBrick + (li >> 6);
            }
            ++base;
        }
    }
}

// ---------------------------------------------------------------------------
// boundary edge extraction: edges bucketed by their smaller vertex
// ---------------------------------------------------------------------------
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
            const unsigned long long pos = voff[a] + (unsigned long long)(atomicSub(&vcnt[a], 1u) - 1u);
            emax[pos] = b;
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

// Per vertex: the other endpoints of its edges; keep those that occur once.
__global__ void edge_find(const unsigned long long *__restrict__ voff, uint32_t *__restrict__ emax, long long nv, uint2 *__restrict__ blist,
                          uint32_t cap, uint32_t *__restrict__ counters)
{
    const long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= nv)
        return;
    const unsigned long long s = voff[a], e = voff[a + 1];
    const long long n = (long long)(e - s);
    if (n == 0)
        return;
    uint32_t *l = emax + s;
    if (n <= 32)
    {
        for (long long i = 0; i < n; ++i)
        {
            int c = 0;
            for (long long j = 0; j < n; ++j)
                c += (l[j] == l[i]);
            if (c == 1)
            {
                const uint32_t slot = atomicAdd(&counters[C_BOUNDARY], 1u);
                if (slot < cap)
                    blist[slot] = make_uint2((uint32_t)a, l[i]);
                else
                    atomicOr(&counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
            }
        }
        return;
    }
    // heap sort in place, then runs of length one
    for (long long i = n / 2 - 1; i >= 0; --i)
        heap_sift(l, i, n);
    for (long long end = n - 1; end > 0; --end)
    {
        const uint32_t t = l[0];
        l[0] = l[end];
        l[end] = t;
        heap_sift(l, 0, end);
    }
    for (long long i = 0; i < n;)
    {
        long long j = i;
        while (j < n && l[j] == l[i])
            ++j;
        if (j - i == 1)
        {
            const uint32_t slot = atomicAdd(&counters[C_BOUNDARY], 1u);
            if (slot < cap)
                blist[slot] = make_uint2((uint32_t)a, l[i]);
            else
                atomicOr(&counters[C_STATUS], (uint32_t)ST_LIST_OVERFLOW);
        }
        i = j;
    }
}

// ---------------------------------------------------------------------------
// per-voxel reduction in reference order + solve
// ---------------------------------------------------------------------------
struct Final
{
    Grid g;
    const float *verts;
    long long nv;
    const void *faces;
    int fbytes;
    float ox, oy, oz;
    float bw, rw;
    const unsigned long long *eseg;
    const unsigned long long *ekey;
    const uint32_t *epay;
    const int32_t *vox;
    float *dual;
    uint8_t *flags;
    uint32_t *counters;
    uint32_t *long_list;
    long long n;
};

struct Acc
{
    float q[10];
    float mean[3];
    float cnt;
    uint32_t flags;
    bool first;
    long long qt_tri;
    float qt[10];
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
    a.qt_tri = -1;
}

__device__ __forceinline__ void tri_q_cached(const Final &F, long long t, Acc &a)
{
    if (a.qt_tri == t)
        return;
    float v[3][3];
    long long idx[3];
    const float o[3] = {F.ox, F.oy, F.oz};
    if (F.fbytes == 8)
        load_triangle<long long>(F.verts, F.nv, (const long long *)F.faces, t, o, v, idx);
    else
        load_triangle<int>(F.verts, F.nv, (const int *)F.faces, t, o, v, idx);
    tri_quadric(v, a.qt);
    a.qt_tri = t;
}

__device__ __forceinline__ void acc_entry(const Final &F, const int vc[3], unsigned long long key, uint32_t pay, Acc &a)
{
    const unsigned stage = (unsigned)(key >> 62);
    if (stage == 0)
    {
        const unsigned sub = (unsigned)(key & 3ull);
        const unsigned long long ta = key >> 2;
        const long long t = (long long)(ta / 3ull);
        const int ax2 = (int)(ta % 3ull);
        const int dx = 1 - (int)(sub & 1u), dy = 1 - (int)(sub >> 1);
        const int ax0 = (ax2 + 1) % 3, ax1 = (ax2 + 2) % 3;
        const int c0 = ax0 == 0 ? vc[0] : (ax0 == 1 ? vc[1] : vc[2]);
        const int c1 = ax1 == 0 ? vc[0] : (ax1 == 1 ? vc[1] : vc[2]);
        const float vs0 = ax0 == 0 ? F.g.vs[0] : (ax0 == 1 ? F.g.vs[1] : F.g.vs[2]);
        const float vs1 = ax1 == 0 ? F.g.vs[0] : (ax1 == 1 ? F.g.vs[1] : F.g.vs[2]);
        const float pu = (float)(c0 - dx + 1) * vs0;
        const float pv = (float)(c1 - dy + 1) * vs1;
        const float pw = __uint_as_float(pay);
        float p[3];
        p[0] = ax2 == 0 ? pw : (ax2 == 1 ? pv : pu);
        p[1] = ax2 == 0 ? pu : (ax2 == 1 ? pw : pv);
        p[2] = ax2 == 0 ? pv : (ax2 == 1 ? pu : pw);
        tri_q_cached(F, t, a);
        if (a.first)
        {
            a.mean[0] = p[0];
            a.mean[1] = p[1];
            a.mean[2] = p[2];
            a.cnt = 1.0f;
#pragma unroll
            for (int i = 0; i < 10; ++i)
                a.q[i] = a.qt[i];
            a.first = false;
        }
        else
        {
            a.mean[0] = a.mean[0] + p[0];
            a.mean[1] = a.mean[1] + p[1];
            a.mean[2] = a.mean[2] + p[2];
            a.cnt = a.cnt + 1.0f;
#pragma unroll
            for (int i = 0; i < 10; ++i)
                a.q[i] = a.q[i] + a.qt[i];
        }
        if (dx == 0 && dy == 0)
            a.flags |= 1u << ax2;
    }
    else if (stage == 1)
    {
        const long long t = (long long)(key & ((1ull << 62) - 1ull));
        tri_q_cached(F, t, a);
#pragma unroll
        for (int i = 0; i < 10; ++i)
            a.q[i] = a.q[i] + a.qt[i];
    }
    else
    {
        const long long ia = (long long)((key >> 31) & 0x7fffffffull);
        const long long ib = (long long)(key & 0x7fffffffull);
        float v0[3], v1[3], bq[10];
        v0[0] = F.verts[ia * 3 + 0] - F.ox;
        v0[1] = F.verts[ia * 3 + 1] - F.oy;
        v0[2] = F.verts[ia * 3 + 2] - F.oz;
        v1[0] = F.verts[ib * 3 + 0] - F.ox;
        v1[1] = F.verts[ib * 3 + 1] - F.oy;
        v1[2] = F.verts[ib * 3 + 2] - F.oz;
        Dda d;
        if (boundary_setup(v0, v1, F.g, d, bq))
        {
#pragma unroll
            for (int i = 0; i < 10; ++i)
                a.q[i] = a.q[i] + F.bw * bq[i];
        }
    }
}

__device__ __forceinline__ void finish_voxel(const Final &F, long long r, const int vc[3], const Acc &a)
{
    float out[3];
    solve_voxel(vc, F.g, a.q, a.mean, a.cnt, F.rw, out);
    F.dual[r * 3 + 0] = out[0];
    F.dual[r * 3 + 1] = out[1];
    F.dual[r * 3 + 2] = out[2];
    F.flags[r * 3 + 0] = (uint8_t)(a.flags & 1u);
    F.flags[r * 3 + 1] = (uint8_t)((a.flags >> 1) & 1u);
    F.flags[r * 3 + 2] = (uint8_t)((a.flags >> 2) & 1u);
}

__global__ void __launch_bounds__(128) final_short(Final F)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= F.n)
        return;
    const unsigned long long s = F.eseg[r];
    const int n = (int)(F.eseg[r + 1] - s);
    if (n > kShortSeg)
    {
        const uint32_t slot = atomicAdd(&F.counters[C_LONG], 1u);
        F.long_list[slot] = (uint32_t)r;
        return;
    }
    unsigned long long k[kShortSeg];
    uint32_t p[kShortSeg];
    for (int i = 0; i < n; ++i)
    {
        const unsigned long long key = F.ekey[s + i];
        const uint32_t pay = F.epay[s + i];
        int j = i;
        while (j > 0 && k[j - 1] > key)
        {
            k[j] = k[j - 1];
            p[j] = p[j - 1];
            --j;
        }
        k[j] = key;
        p[j] = pay;
    }
    const int vc[3] = {F.vox[r * 3 + 0], F.vox[r * 3 + 1], F.vox[r * 3 + 2]};
    Acc a;
    acc_init(a);
    for (int i = 0; i < n; ++i)
        acc_entry(F, vc, k[i], p[i], a);
    finish_voxel(F, r, vc, a);
}

// One CTA per voxel with more than kShortSeg contributions.
__global__ void __launch_bounds__(128) final_long(Final F)
{
    __shared__ unsigned long long skey[kLongSmem];
    __shared__ uint32_t spay[kLongSmem];
    __shared__ uint16_t sperm[kLongSmem];
    const uint32_t nl = F.counters[C_LONG];
    for (uint32_t li = blockIdx.x; li < nl; li += gridDim.x)
    {
        const long long r = F.long_list[li];
        const unsigned long long s = F.eseg[r];
        const long long n = (long long)(F.eseg[r + 1] - s);
        const int vc[3] = {F.vox[r * 3 + 0], F.vox[r * 3 + 1], F.vox[r * 3 + 2]};
        if (n <= kLongSmem)
        {
            for (long long i = threadIdx.x; i < n; i += blockDim.x)
            {
                skey[i] = F.ekey[s + i];
                spay[i] = F.epay[s + i];
            }
            __syncthreads();
            for (long long i = threadIdx.x; i < n; i += blockDim.x)
            {
                const unsigned long long ki = skey[i];
                int rank = 0;
                for (long long j = 0; j < n; ++j)
                    rank += (skey[j] < ki) || (skey[j] == ki && j < i);
                sperm[rank] = (uint16_t)i;
            }
            __syncthreads();
            if (threadIdx.x == 0)
            {
                Acc a;
                acc_init(a);
                for (long long i = 0; i < n; ++i)
                    acc_entry(F, vc, skey[sperm[i]], spay[sperm[i]], a);
                finish_voxel(F, r, vc, a);
            }
            __syncthreads();
        }
        else if (threadIdx.x == 0)
        {
            // very long segment: repeated selection of the next key (keys are unique per voxel)
            Acc a;
            acc_init(a);
            unsigned long long last = 0;
            for (long long step = 0; step < n; ++step)
            {
                unsigned long long best = ~0ull;
                uint32_t bp = 0;
                for (long long j = 0; j < n; ++j)
                {
                    const unsigned long long kj = F.ekey[s + j];
                    if ((step == 0 || kj > last) && kj <= best)
                    {
                        best = kj;
                        bp = F.epay[s + j];
                    }
                }
                acc_entry(F, vc, best, bp, a);
                last = best;
            }
            finish_voxel(F, r, vc, a);
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
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
    Buf bits, bcount, bbase, word_base, counters, scan_large, face_large;
    Buf vcnt, voff, emax, blist;
    Buf ecount, eseg, ekey, epay, long_list, cub_tmp;
    unsigned long long *host = nullptr; // pinned readback words
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
    long long n_vox = 0;
};

namespace
{

int fail(ovx_fdg_context *c, int status, const char *what)
{
    if (c)
        c->err = what;
    return status;
}

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

cudaError_t ensure(Buf &b, size_t bytes)
{
    if (bytes == 0)
        bytes = 16;
    if (b.cap >= bytes)
        return cudaSuccess;
    if (b.p)
    {
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    const size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess)
    {
        cudaGetLastError();
        b.p = nullptr;
        return e;
    }
    b.cap = want;
    return cudaSuccess;
}

template <typename In, typename Out>
cudaError_t exclusive_scan(ovx_fdg_context *ctx, const In *in, Out *out, long long n, cudaStream_t st)
{
    size_t bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveScan(nullptr, bytes, in, out, cub::Sum(), Out(0), (int)n, st);
    if (e != cudaSuccess)
        return e;
    e = ensure(ctx->cub_tmp, bytes);
    if (e != cudaSuccess)
        return e;
    return cub::DeviceScan::ExclusiveScan(ctx->cub_tmp.p, bytes, in, out, cub::Sum(), Out(0), (int)n, st);
}

inline unsigned blocks_for(long long n, int threads)
{
    return (unsigned)((n + threads - 1) / threads);
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
        g.gmin[a] = grid->grid_min[a];
        g.gmax[a] = grid->grid_max[a];
        const long long sz = (long long)grid->grid_max[a] - (long long)grid->grid_min[a];
        if (sz < 1 || sz > (1 << 20))
            return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "grid_range must satisfy 1 <= grid_max - grid_min <= 2^20");
        g.size[a] = (int)sz;
        g.nb[a] = (int)((sz + kBrick - 1) / kBrick);
        nb *= g.nb[a];
    }
    if (nb * kWordsPerBrick * 4ll > (64ll << 30))
        return fail(ctx, OVX_FDG_CAPACITY, "grid too large for the dense brick bitmap (64 GiB limit)");
    g.nbricks = nb;
    return OVX_FDG_OK;
}

template <typename IdxT>
void launch_mark(Pass &P, cudaStream_t st, int sms)
{
    if (P.nf > 0)
        tri_pass<MARK, IdxT><<<blocks_for(P.nf, kThreads), kThreads, 0, st>>>(P);
    large_scan<MARK, IdxT><<<sms * 4, 128, 0, st>>>(P);
}

template <int M, typename IdxT>
void launch_replay(Pass &P, cudaStream_t st, int sms, bool boundary)
{
    if (P.nf > 0)
        tri_pass<M, IdxT><<<blocks_for(P.nf, kThreads), kThreads, 0, st>>>(P);
    large_scan<M, IdxT><<<sms * 4, 128, 0, st>>>(P);
    if (P.face_on)
        large_face<M, IdxT><<<sms * 4, 128, 0, st>>>(P);
    if (boundary)
        boundary_pass<M><<<sms * 8, kThreads, 0, st>>>(P);
}

Pass make_pass(ovx_fdg_context *c)
{
    Pass P{};
    P.g = c->g;
    P.verts = c->verts;
    P.nv = c->nv;
    P.faces = c->faces;
    P.nf = c->nf;
    P.ox = c->origin[0];
    P.oy = c->origin[1];
    P.oz = c->origin[2];
    P.bits = (uint32_t *)c->bits.p;
    P.word_base = (const uint32_t *)c->word_base.p;
    P.ecount = (uint32_t *)c->ecount.p;
    P.eseg = (const unsigned long long *)c->eseg.p;
    P.ekey = (unsigned long long *)c->ekey.p;
    P.epay = (uint32_t *)c->epay.p;
    P.counters = (uint32_t *)c->counters.p;
    P.scan_large = (uint32_t *)c->scan_large.p;
    P.scan_large_cap = (uint32_t)(c->scan_large.cap / 4 < 0xffffffffull ? c->scan_large.cap / 4 : 0xffffffffull);
    P.face_large = (uint32_t *)c->face_large.p;
    P.face_large_cap = (uint32_t)(c->face_large.cap / 4 < 0xffffffffull ? c->face_large.cap / 4 : 0xffffffffull);
    P.blist = (const uint2 *)c->blist.p;
    P.blist_cap = (uint32_t)(c->blist.cap / 8 < 0xffffffffull ? c->blist.cap / 8 : 0xffffffffull);
    P.face_on = c->fw > 0.0f ? 1 : 0;
    return P;
}

int status_to_error(ovx_fdg_context *ctx, uint32_t st)
{
    if (st & ST_BAD_INDEX)
        return fail(ctx, OVX_FDG_BAD_FACE_INDEX, "face index out of range [0, num_vertices)");
    if (st & ST_LIST_OVERFLOW)
        return fail(ctx, OVX_FDG_INTERNAL, "work list overflow");
    if (st & ST_REPLAY)
        return fail(ctx, OVX_FDG_INTERNAL, "contribution replay mismatch");
    if (st & ST_WALK_GUARD)
        return fail(ctx, OVX_FDG_INTERNAL, "boundary walk exceeded its step bound (non-finite vertex?)");
    return OVX_FDG_OK;
}

// Occupancy stage shared by the full conversion and intersect_occ.
int occupancy_stage(ovx_fdg_context *ctx, cudaStream_t st, bool with_boundary, int64_t *num_voxels)
{
    const Grid &g = ctx->g;
    const long long nf = ctx->nf;
    OVX_CUDA(ensure(ctx->bits, (size_t)g.nbricks * kWordsPerBrick * 4));
    OVX_CUDA(ensure(ctx->bcount, (size_t)(g.nbricks + 1) * 4));
    OVX_CUDA(ensure(ctx->bbase, (size_t)(g.nbricks + 1) * 8));
    OVX_CUDA(ensure(ctx->counters, C_WORDS * 4));
    OVX_CUDA(ensure(ctx->scan_large, (size_t)(3 * nf + 1) * 4));
    OVX_CUDA(ensure(ctx->face_large, (size_t)(nf + 1) * 4));
    if (with_boundary)
    {
        OVX_CUDA(ensure(ctx->vcnt, (size_t)(ctx->nv + 1) * 4));
        OVX_CUDA(ensure(ctx->voff, (size_t)(ctx->nv + 1) * 8));
        OVX_CUDA(ensure(ctx->emax, (size_t)(3 * nf + 1) * 4));
        OVX_CUDA(ensure(ctx->blist, (size_t)(3 * nf + 1) * 8));
    }
    OVX_CUDA(cudaMemsetAsync(ctx->bits.p, 0, (size_t)g.nbricks * kWordsPerBrick * 4, st));
    OVX_CUDA(cudaMemsetAsync(ctx->counters.p, 0, C_WORDS * 4, st));
    OVX_CUDA(cudaMemsetAsync((uint32_t *)ctx->bcount.p + g.nbricks, 0, 4, st));

    Pass P = make_pass(ctx);
    if (ctx->fbytes == 8)
        launch_mark<long long>(P, st, ctx->sms);
    else
        launch_mark<int>(P, st, ctx->sms);
    OVX_CUDA(cudaGetLastError());

    brick_count<<<blocks_for(g.nbricks, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->bits.p, g.nbricks,
                                                                      (uint32_t *)ctx->bcount.p);
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->bcount.p, (unsigned long long *)ctx->bbase.p, g.nbricks + 1, st));

    if (with_boundary && nf > 0)
    {
        OVX_CUDA(cudaMemsetAsync(ctx->vcnt.p, 0, (size_t)(ctx->nv + 1) * 4, st));
        uint32_t *vcnt = (uint32_t *)ctx->vcnt.p;
        unsigned long long *voff = (unsigned long long *)ctx->voff.p;
        if (ctx->fbytes == 8)
            edge_count<long long><<<blocks_for(nf, kThreads), kThreads, 0, st>>>((const long long *)ctx->faces, nf, ctx->nv, vcnt);
        else
            edge_count<int><<<blocks_for(nf, kThreads), kThreads, 0, st>>>((const int *)ctx->faces, nf, ctx->nv, vcnt);
        OVX_CUDA(cudaGetLastError());
        OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)vcnt, voff, ctx->nv + 1, st));
        if (ctx->fbytes == 8)
            edge_fill<long long><<<blocks_for(nf, kThreads), kThreads, 0, st>>>((const long long *)ctx->faces, nf, ctx->nv, voff, vcnt,
                                                                               (uint32_t *)ctx->emax.p);
        else
            edge_fill<int><<<blocks_for(nf, kThreads), kThreads, 0, st>>>((const int *)ctx->faces, nf, ctx->nv, voff, vcnt,
                                                                         (uint32_t *)ctx->emax.p);
        OVX_CUDA(cudaGetLastError());
        if (ctx->nv > 0)
            edge_find<<<blocks_for(ctx->nv, kThreads), kThreads, 0, st>>>(voff, (uint32_t *)ctx->emax.p, ctx->nv, (uint2 *)ctx->blist.p,
                                                                         P.blist_cap, (uint32_t *)ctx->counters.p);
        OVX_CUDA(cudaGetLastError());
    }

    OVX_CUDA(cudaMemcpyAsync(&ctx->host[0], (unsigned long long *)ctx->bbase.p + g.nbricks, 8, cudaMemcpyDeviceToHost, st));
    OVX_CUDA(cudaMemcpyAsync(&ctx->host[1], ctx->counters.p, C_WORDS * 4, cudaMemcpyDeviceToHost, st));
    OVX_CUDA(cudaStreamSynchronize(st));
    const uint32_t *hc = (const uint32_t *)&ctx->host[1];
    const int rc = status_to_error(ctx, hc[C_STATUS]);
    if (rc != OVX_FDG_OK)
        return rc;
    const unsigned long long n = ctx->host[0];
    if (n >= (1ull << 31))
        return fail(ctx, OVX_FDG_CAPACITY, "more than 2^31-1 occupied voxels");
    ctx->n_vox = (long long)n;
    *num_voxels = (int64_t)n;
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
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaMallocHost((void **)&ctx->host, 16 * sizeof(unsigned long long));
    cudaSetDevice(prev);
    if (e != cudaSuccess)
    {
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
    Buf *all[] = {&ctx->bits, &ctx->bcount, &ctx->bbase, &ctx->word_base, &ctx->counters, &ctx->scan_large, &ctx->face_large,
                  &ctx->vcnt, &ctx->voff, &ctx->emax, &ctx->blist, &ctx->ecount, &ctx->eseg, &ctx->ekey, &ctx->epay,
                  &ctx->long_list, &ctx->cub_tmp};
    for (Buf *b : all)
        if (b->p)
            cudaFree(b->p);
    if (ctx->host)
        cudaFreeHost(ctx->host);
    cudaSetDevice(prev);
    delete ctx;
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
    const Buf *all[] = {&ctx->bits, &ctx->bcount, &ctx->bbase, &ctx->word_base, &ctx->counters, &ctx->scan_large, &ctx->face_large,
                        &ctx->vcnt, &ctx->voff, &ctx->emax, &ctx->blist, &ctx->ecount, &ctx->eseg, &ctx->ekey, &ctx->epay,
                        &ctx->long_list, &ctx->cub_tmp};
    int64_t s = 0;
    for (const Buf *b : all)
        s += (int64_t)b->cap;
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
    if (num_faces >= (1ll << 30) || num_vertices >= (1ll << 31) - 1)
        return fail(ctx, OVX_FDG_CAPACITY, "more than 2^30 faces or 2^31-1 vertices");
    Grid g{};
    int rc = check_grid(ctx, grid, g);
    if (rc != OVX_FDG_OK)
        return rc;
    OVX_CUDA(cudaSetDevice(ctx->device));
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
    rc = occupancy_stage(ctx, (cudaStream_t)stream, boundary_weight > 0.0f, num_voxels);
    if (rc != OVX_FDG_OK)
        return rc;
    ctx->phase = 1;
    return OVX_FDG_OK;
}

int ovx_fdg_finish(ovx_fdg_context *ctx, void *stream, int32_t *voxel_indices, float *dual_vertices, uint8_t *intersected)
{
    if (!ctx)
        return OVX_FDG_INVALID_ARGUMENT;
    if (ctx->phase != 1)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "ovx_fdg_finish without a successful ovx_fdg_begin");
    ctx->phase = 0;
    const long long n = ctx->n_vox;
    if (n == 0)
        return OVX_FDG_OK;
    if (!voxel_indices || !dual_vertices || !intersected)
        return fail(ctx, OVX_FDG_INVALID_ARGUMENT, "NULL output buffer");
    cudaStream_t st = (cudaStream_t)stream;
    OVX_CUDA(cudaSetDevice(ctx->device));
    const Grid &g = ctx->g;
    OVX_CUDA(ensure(ctx->word_base, (size_t)g.nbricks * kWordsPerBrick * 4));
    OVX_CUDA(ensure(ctx->ecount, (size_t)(n + 1) * 4));
    OVX_CUDA(ensure(ctx->eseg, (size_t)(n + 1) * 8));
    OVX_CUDA(ensure(ctx->long_list, (size_t)(n + 1) * 4));

    brick_emit<<<blocks_for(g.nbricks, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->bits.p,
                                                                     (const unsigned long long *)ctx->bbase.p, g,
                                                                     (uint32_t *)ctx->word_base.p, voxel_indices);
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(cudaMemsetAsync(ctx->ecount.p, 0, (size_t)(n + 1) * 4, st));

    const bool boundary = ctx->bw > 0.0f;
    Pass P = make_pass(ctx);
    if (ctx->fbytes == 8)
        launch_replay<COUNT, long long>(P, st, ctx->sms, boundary);
    else
        launch_replay<COUNT, int>(P, st, ctx->sms, boundary);
    OVX_CUDA(cudaGetLastError());
    OVX_CUDA(exclusive_scan(ctx, (const uint32_t *)ctx->ecount.p, (unsigned long long *)ctx->eseg.p, n + 1, st));
    OVX_CUDA(cudaMemcpyAsync(&ctx->host[0], (unsigned long long *)ctx->eseg.p + n, 8, cudaMemcpyDeviceToHost, st));
    OVX_CUDA(cudaMemcpyAsync(&ctx->host[1], ctx->counters.p, C_WORDS * 4, cudaMemcpyDeviceToHost, st));
    OVX_CUDA(cudaStreamSynchronize(st));
    int rc = status_to_error(ctx, ((const uint32_t *)&ctx->host[1])[C_STATUS]);
    if (rc != OVX_FDG_OK)
        return rc;
    const unsigned long long E = ctx->host[0];
    OVX_CUDA(ensure(ctx->ekey, (size_t)E * 8));
    OVX_CUDA(ensure(ctx->epay, (size_t)E * 4));

    P = make_pass(ctx);
    if (ctx->fbytes == 8)
        launch_replay<FILL, long long>(P, st, ctx->sms, boundary);
    else
        launch_replay<FILL, int>(P, st, ctx->sms, boundary);
    OVX_CUDA(cudaGetLastError());

    Final F{};
    F.g = g;
    F.verts = ctx->verts;
    F.nv = ctx->nv;
    F.faces = ctx->faces;
    F.fbytes = ctx->fbytes;
    F.ox = ctx->origin[0];
    F.oy = ctx->origin[1];
    F.oz = ctx->origin[2];
    F.bw = ctx->bw;
    F.rw = ctx->rw;
    F.eseg = (const unsigned long long *)ctx->eseg.p;
    F.ekey = (const unsigned long long *)ctx->ekey.p;
    F.epay = (const uint32_t *)ctx->epay.p;
    F.vox = voxel_indices;
    F.dual = dual_vertices;
    F.flags = intersected;
    F.counters = (uint32_t *)ctx->counters.p;
    F.long_list = (uint32_t *)ctx->long_list.p;
    F.n = n;
    final_short<<<blocks_for(n, 128), 128, 0, st>>>(F);
    final_long<<<ctx->sms * 2, 128, 0, st>>>(F);
    OVX_CUDA(cudaGetLastError());
    return OVX_FDG_OK;
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
    OVX_CUDA(cudaSetDevice(ctx->device));
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
    OVX_CUDA(cudaSetDevice(ctx->device));
    brick_emit<<<blocks_for(ctx->g.nbricks, kThreads), kThreads, 0, st>>>((const uint32_t *)ctx->bits.p,
                                                                          (const unsigned long long *)ctx->bbase.p, ctx->g,
                                                                          nullptr, voxel_indices);
    OVX_CUDA(cudaGetLastError());
    return OVX_FDG_OK;
}

} // extern "C"
