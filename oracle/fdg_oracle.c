/*
 * fdg_oracle.c -- CPU oracle for mesh -> flexible dual grid.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against (tests, smoke check, and the CPU-baseline leg of the benchmark).  The
 * product never links, loads or calls it.
 *
 * It restates, in plain C, the reference CPU implementation
 * (src/convert/flexible_dual_grid.cpp of quantaji/o-voxel-gpu) with every
 * floating-point operation written out in a fixed order:
 *   - no FMA contraction (build with -ffp-contract=off; x86-64 baseline has no FMA),
 *   - fixed-size Eigen reductions as the SSE2 build evaluates them:
 *       3 floats  a0*b0 + (a1*b1 + a2*b2)
 *       4 floats  (a0*b0 + a2*b2) + (a1*b1 + a3*b3)     (one packet, predux)
 *       3 doubles (a0*b0 + a1*b1) + a2*b2               (one Packet2d + tail)
 *       runtime-sized reductions left to right,
 *   - float->int conversions with x86 cvtt semantics (out of range -> INT_MIN).
 * Eigen itself is not present (it is an un-vendored submodule of the
 * reference), so these orders are this project's reading of Eigen 3.4's
 * published evaluator design; they are pinned against the reference source
 * compiled with the project's Eigen-API shim (oracle/eigen_shim), not against
 * real Eigen.
 *
 * Entry points (ctypes):
 *   fdg_oracle_mesh_to_fdg_f32  exact restatement (float accumulation, float solve)
 *   fdg_oracle_mesh_to_fdg_f64  same geometry decisions, FP64 quadrics/accumulation/solve
 *   fdg_oracle_intersect_occ    occupancy only (flexible_dual_grid.cpp:80-156)
 *   fdg_oracle_free
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define FDG_ORACLE_BAD_INDEX 2
#define FDG_ORACLE_OOM 3

typedef struct fdg_oracle_out
{
    int64_t num_voxels;
    int32_t *voxels;      /* [N,3] insertion order (first event that touched the voxel) */
    void *dual;           /* [N,3] REAL */
    uint8_t *intersected; /* [N,3] */
    void *qef;            /* [N,10] REAL, intersection+face+boundary quadric before regularisation */
    void *mean_sum;       /* [N,3] REAL */
    void *cnt;            /* [N] REAL */
    int64_t num_boundary_edges;
    int32_t elem_size; /* sizeof(REAL) */
    int32_t pad;
} fdg_oracle_out;

/* ---------------- x86 conversion semantics ---------------- */
static inline int trunc_d2i(double d)
{
    return (d > -2147483649.0 && d < 2147483648.0) ? (int)d : INT_MIN;
}
static inline int trunc_f2i(float f)
{
    return (f > -2147483904.0f && f < 2147483648.0f) ? (int)f : INT_MIN;
}
static inline int clampi(int v, int lo, int hi)
{
    /* std::clamp(v, lo, hi) */
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
static inline float dot3f(float a0, float a1, float a2, float b0, float b1, float b2)
{
    return a0 * b0 + (a1 * b1 + a2 * b2);
}
static inline float dot2f(float a0, float a1, float b0, float b1)
{
    return a0 * b0 + a1 * b1;
}
static inline float maxf0(float a)
{
    /* std::max(a, 0.0f) as Eigen's cwiseMax(0.0f) evaluates it */
    return (a < 0.0f) ? 0.0f : a;
}

/* Triangle normal: normalize(cross(v1 - v0, v2 - v1)) in float, Eigen normalized() semantics. */
static void tri_normal(const float v[3][3], float n[3])
{
    const float e0[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
    const float e1[3] = {v[2][0] - v[1][0], v[2][1] - v[1][1], v[2][2] - v[1][2]};
    n[0] = e0[1] * e1[2] - e0[2] * e1[1];
    n[1] = e0[2] * e1[0] - e0[0] * e1[2];
    n[2] = e0[0] * e1[1] - e0[1] * e1[0];
    const float s = dot3f(n[0], n[1], n[2], n[0], n[1], n[2]);
    if (s > 0.0f)
    {
        const float r = sqrtf(s);
        n[0] = n[0] / r;
        n[1] = n[1] / r;
        n[2] = n[2] / r;
    }
}

/* FP64 variant of the normal (used only by the FP64 oracle build). */
static void tri_normal_f64(const float v[3][3], double n[3])
{
    const double e0[3] = {(double)v[1][0] - v[0][0], (double)v[1][1] - v[0][1], (double)v[1][2] - v[0][2]};
    const double e1[3] = {(double)v[2][0] - v[1][0], (double)v[2][1] - v[1][1], (double)v[2][2] - v[1][2]};
    n[0] = e0[1] * e1[2] - e0[2] * e1[1];
    n[1] = e0[2] * e1[0] - e0[0] * e1[2];
    n[2] = e0[0] * e1[1] - e0[1] * e1[0];
    const double s = n[0] * n[0] + (n[1] * n[1] + n[2] * n[2]);
    if (s > 0.0)
    {
        const double r = sqrt(s);
        n[0] /= r;
        n[1] /= r;
        n[2] /= r;
    }
}

/* ---------------- voxel hash map (coordinate -> insertion index) ---------------- */
typedef struct vox_map
{
    uint64_t *keys; /* 0 = empty; stored key = packed + 1 */
    int64_t *vals;
    uint64_t cap;
    uint64_t count;
} vox_map;

static int32_t g_gmin[3], g_gmax[3];
static void map_set_grid(const int32_t gmin[3], const int32_t gmax[3])
{
    memcpy(g_gmin, gmin, sizeof(g_gmin));
    memcpy(g_gmax, gmax, sizeof(g_gmax));
}
static inline uint64_t map_key(const int32_t c[3])
{
    const uint64_t sx = (uint64_t)(int64_t)(g_gmax[0] - g_gmin[0]);
    const uint64_t sy = (uint64_t)(int64_t)(g_gmax[1] - g_gmin[1]);
    return (uint64_t)(int64_t)(c[0] - g_gmin[0]) + sx * ((uint64_t)(int64_t)(c[1] - g_gmin[1]) + sy * (uint64_t)(int64_t)(c[2] - g_gmin[2]));
}
static inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 31;
    x *= 0x7fb5d329728ea185ULL;
    x ^= x >> 27;
    x *= 0x81dadef4bc2dd44dULL;
    x ^= x >> 33;
    return x;
}
static int map_init(vox_map *m, uint64_t cap)
{
    m->cap = cap;
    m->count = 0;
    m->keys = (uint64_t *)calloc(cap, sizeof(uint64_t));
    m->vals = (int64_t *)malloc(cap * sizeof(int64_t));
    return (m->keys && m->vals) ? 0 : -1;
}
static void map_free(vox_map *m)
{
    free(m->keys);
    free(m->vals);
    m->keys = NULL;
    m->vals = NULL;
}
static int64_t map_find(const vox_map *m, uint64_t key)
{
    const uint64_t k = key + 1;
    uint64_t s = mix64(k) & (m->cap - 1);
    for (;;)
    {
        const uint64_t f = m->keys[s];
        if (f == 0)
            return -1;
        if (f == k)
            return m->vals[s];
        s = (s + 1) & (m->cap - 1);
    }
}
static int map_insert(vox_map *m, uint64_t key, int64_t val);
static int map_grow(vox_map *m)
{
    vox_map n;
    if (map_init(&n, m->cap * 2) != 0)
        return -1;
    for (uint64_t i = 0; i < m->cap; ++i)
        if (m->keys[i])
            map_insert(&n, m->keys[i] - 1, m->vals[i]);
    map_free(m);
    *m = n;
    return 0;
}
static int map_insert(vox_map *m, uint64_t key, int64_t val)
{
    if ((m->count + 1) * 2 > m->cap)
        if (map_grow(m) != 0)
            return -1;
    const uint64_t k = key + 1;
    uint64_t s = mix64(k) & (m->cap - 1);
    while (m->keys[s] != 0 && m->keys[s] != k)
        s = (s + 1) & (m->cap - 1);
    if (m->keys[s] == 0)
        m->count++;
    m->keys[s] = k;
    m->vals[s] = val;
    return 0;
}

/* ---------------- scanline events (flexible_dual_grid.cpp:195-283) ---------------- */
typedef void (*event_fn)(void *ctx, const int32_t coord[3], int ax2, int dx, int dy, const double pt[3]);

static inline void lerp2(double a, double b, double t, double va0, double va1, double vb0, double vb1,
                         double *r0, double *r1)
{
    if (a == b)
    {
        *r0 = va0;
        *r1 = va1;
        return;
    }
    const double alpha = (t - a) / (b - a);
    const double oma = 1.0 - alpha;
    *r0 = oma * va0 + alpha * vb0;
    *r1 = oma * va1 + alpha * vb1;
}
static inline double lerp1(double a, double b, double t, double va, double vb)
{
    if (a == b)
        return va;
    const double alpha = (t - a) / (b - a);
    return (1.0 - alpha) * va + alpha * vb;
}

static void scan_half(int row_start, int row_end, const double T0[3], const double T1[3], const double T2[3],
                      int ax0, int ax1, int ax2, const float vs[3], const int32_t gmin[3], const int32_t gmax[3],
                      event_fn fn, void *ctx)
{
    for (int yi = row_start; yi < row_end; ++yi)
    {
        const double y = (double)((float)(yi + 1) * vs[ax1]);
        double t3x, t3z, t4x, t4z;
        lerp2(T0[1], T1[1], y, T0[0], T0[2], T1[0], T1[2], &t3x, &t3z);
        lerp2(T0[1], T2[1], y, T0[0], T0[2], T2[0], T2[2], &t4x, &t4z);
        if (t3x > t4x)
        {
            double t = t3x; t3x = t4x; t4x = t;
            t = t3z; t3z = t4z; t4z = t;
        }
        const int ls = clampi(trunc_d2i(t3x / (double)vs[ax0]), gmin[ax0], gmax[ax0] - 1);
        const int le = clampi(trunc_d2i(t4x / (double)vs[ax0]), gmin[ax0], gmax[ax0] - 1);
        for (int xi = ls; xi < le; ++xi)
        {
            const double x = (double)((float)(xi + 1) * vs[ax0]);
            const double z = lerp1(t3x, t4x, x, t3z, t4z);
            const int zi = trunc_d2i(z / (double)vs[ax2]);
            if (zi >= gmin[ax2] && zi < gmax[ax2])
            {
                for (int dx = 0; dx < 2; ++dx)
                    for (int dy = 0; dy < 2; ++dy)
                    {
                        int32_t c[3];
                        double pt[3];
                        c[ax0] = xi + dx;
                        c[ax1] = yi + dy;
                        c[ax2] = zi;
                        pt[ax0] = x;
                        pt[ax1] = y;
                        pt[ax2] = z;
                        fn(ctx, c, ax2, dx, dy, pt);
                    }
            }
        }
    }
}

static void scan_triangle(const float v[3][3], const float vs[3], const int32_t gmin[3], const int32_t gmax[3],
                          event_fn fn, void *ctx)
{
    for (int ax2 = 0; ax2 < 3; ++ax2)
    {
        const int ax0 = (ax2 + 1) % 3, ax1 = (ax2 + 2) % 3;
        double t[3][3];
        for (int k = 0; k < 3; ++k)
        {
            t[k][0] = v[k][ax0];
            t[k][1] = v[k][ax1];
            t[k][2] = v[k][ax2];
        }
        /* libstdc++ std::sort on 3 elements = insertion sort (stable) with comparator a.y < b.y */
        for (int i = 1; i < 3; ++i)
        {
            double val[3] = {t[i][0], t[i][1], t[i][2]};
            if (val[1] < t[0][1])
            {
                for (int j = i; j > 0; --j)
                    memcpy(t[j], t[j - 1], sizeof(t[0]));
                memcpy(t[0], val, sizeof(val));
            }
            else
            {
                int j = i;
                while (val[1] < t[j - 1][1])
                {
                    memcpy(t[j], t[j - 1], sizeof(t[0]));
                    --j;
                }
                memcpy(t[j], val, sizeof(val));
            }
        }
        const int start = clampi(trunc_d2i(t[0][1] / (double)vs[ax1]), gmin[ax1], gmax[ax1] - 1);
        const int mid = clampi(trunc_d2i(t[1][1] / (double)vs[ax1]), gmin[ax1], gmax[ax1] - 1);
        const int end = clampi(trunc_d2i(t[2][1] / (double)vs[ax1]), gmin[ax1], gmax[ax1] - 1);
        scan_half(start, mid, t[0], t[1], t[2], ax0, ax1, ax2, vs, gmin, gmax, fn, ctx);
        scan_half(mid, end, t[2], t[1], t[0], ax0, ax1, ax2, vs, gmin, gmax, fn, ctx);
    }
}

/* ---------------- face stage predicates (flexible_dual_grid.cpp:304-402) ---------------- */
typedef struct face_setup
{
    float n[3];
    float d1, d2;
    float nxy[3][2], dxy[3];
    float nyz[3][2], dyz[3];
    float nzx[3][2], dzx[3];
    int bmin[3], bmax[3];
} face_setup;

static void face_prepare(const float v[3][3], const float vs[3], const int32_t gmin[3], const int32_t gmax[3],
                         face_setup *fs)
{
    const float e[3][3] = {
        {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]},
        {v[2][0] - v[1][0], v[2][1] - v[1][1], v[2][2] - v[1][2]},
        {v[0][0] - v[2][0], v[0][1] - v[2][1], v[0][2] - v[2][2]}};
    tri_normal(v, fs->n);
    const float *n = fs->n;
    for (int i = 0; i < 3; ++i)
    {
        float mn = v[0][i], mx = v[0][i];
        /* cwiseMin / cwiseMax chain: std::min(a,b) = (b < a) ? b : a */
        mn = (v[1][i] < mn) ? v[1][i] : mn;
        mn = (v[2][i] < mn) ? v[2][i] : mn;
        mx = (mx < v[1][i]) ? v[1][i] : mx;
        mx = (mx < v[2][i]) ? v[2][i] : mx;
        const float lo = mn / vs[i], hi = mx / vs[i];
        const int l = trunc_f2i(lo);
        const int h = trunc_f2i(hi + 1.0f);
        fs->bmin[i] = (l < gmin[i]) ? gmin[i] : l;
        fs->bmax[i] = (gmax[i] < h) ? gmax[i] : h;
    }
    const float c[3] = {n[0] > 0.0f ? vs[0] : 0.0f, n[1] > 0.0f ? vs[1] : 0.0f, n[2] > 0.0f ? vs[2] : 0.0f};
    fs->d1 = dot3f(n[0], n[1], n[2], c[0] - v[0][0], c[1] - v[0][1], c[2] - v[0][2]);
    fs->d2 = dot3f(n[0], n[1], n[2], (vs[0] - c[0]) - v[0][0], (vs[1] - c[1]) - v[0][1], (vs[2] - c[2]) - v[0][2]);

    const float mxy = (n[2] < 0.0f) ? -1.0f : 1.0f;
    const float myz = (n[0] < 0.0f) ? -1.0f : 1.0f;
    const float mzx = (n[1] < 0.0f) ? -1.0f : 1.0f;
    for (int k = 0; k < 3; ++k)
    {
        const float *vk = v[k];
        /* XY: n = (-m*e.y, m*e.x), vertex (x, y), extent (vs.x, vs.y) */
        fs->nxy[k][0] = (-mxy) * e[k][1];
        fs->nxy[k][1] = mxy * e[k][0];
        fs->dxy[k] = -dot2f(fs->nxy[k][0], fs->nxy[k][1], vk[0], vk[1]) +
                     dot2f(maxf0(fs->nxy[k][0]), maxf0(fs->nxy[k][1]), vs[0], vs[1]);
        /* YZ: n = (-m*e.z, m*e.y), vertex (y, z), extent (vs.y, vs.z) */
        fs->nyz[k][0] = (-myz) * e[k][2];
        fs->nyz[k][1] = myz * e[k][1];
        fs->dyz[k] = -dot2f(fs->nyz[k][0], fs->nyz[k][1], vk[1], vk[2]) +
                     dot2f(maxf0(fs->nyz[k][0]), maxf0(fs->nyz[k][1]), vs[1], vs[2]);
        /* ZX: n = (-m*e.x, m*e.z), vertex (z, x), extent (vs.z, vs.x) */
        fs->nzx[k][0] = (-mzx) * e[k][0];
        fs->nzx[k][1] = mzx * e[k][2];
        fs->dzx[k] = -dot2f(fs->nzx[k][0], fs->nzx[k][1], vk[2], vk[0]) +
                     dot2f(maxf0(fs->nzx[k][0]), maxf0(fs->nzx[k][1]), vs[2], vs[0]);
    }
}

static int face_test(const face_setup *fs, const float vs[3], int x, int y, int z)
{
    const float p[3] = {vs[0] * (float)x, vs[1] * (float)y, vs[2] * (float)z};
    const float nd = dot3f(fs->n[0], fs->n[1], fs->n[2], p[0], p[1], p[2]);
    if ((nd + fs->d1) * (nd + fs->d2) > 0.0f)
        return 0;
    for (int k = 0; k < 3; ++k)
        if (dot2f(fs->nxy[k][0], fs->nxy[k][1], p[0], p[1]) + fs->dxy[k] < 0.0f)
            return 0;
    for (int k = 0; k < 3; ++k)
        if (dot2f(fs->nyz[k][0], fs->nyz[k][1], p[1], p[2]) + fs->dyz[k] < 0.0f)
            return 0;
    for (int k = 0; k < 3; ++k)
        if (dot2f(fs->nzx[k][0], fs->nzx[k][1], p[2], p[0]) + fs->dzx[k] < 0.0f)
            return 0;
    return 1;
}

/* ---------------- boundary edges (flexible_dual_grid.cpp:728-756) ---------------- */
static int cmp_u64(const void *a, const void *b)
{
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}
/* Returns undirected edges (min<<32 | max) used by exactly one face, ascending. */
static uint64_t *boundary_edges(const int32_t *faces, int64_t nf, int64_t *ne)
{
    *ne = 0;
    if (nf == 0)
        return NULL;
    uint64_t *e = (uint64_t *)malloc((size_t)nf * 3 * sizeof(uint64_t));
    if (!e)
        return NULL;
    for (int64_t f = 0; f < nf; ++f)
        for (int k = 0; k < 3; ++k)
        {
            int32_t a = faces[f * 3 + k], b = faces[f * 3 + (k + 1) % 3];
            if (a > b)
            {
                int32_t t = a; a = b; b = t;
            }
            e[f * 3 + k] = ((uint64_t)(uint32_t)a << 32) | (uint32_t)b;
        }
    qsort(e, (size_t)nf * 3, sizeof(uint64_t), cmp_u64);
    int64_t out = 0;
    for (int64_t i = 0; i < nf * 3;)
    {
        int64_t j = i;
        while (j < nf * 3 && e[j] == e[i])
            ++j;
        if (j - i == 1)
            e[out++] = e[i];
        i = j;
    }
    *ne = out;
    return e;
}

/* ---------------- boundary quadric + DDA (flexible_dual_grid.cpp:427-507) ---------------- */
typedef struct dda_state
{
    int32_t cur[3];
    int32_t step[3];
    double tmax[3], tdelta[3];
    double len;
    int started;
    int64_t guard;
} dda_state;

/* Returns 0 when the segment is skipped (length < 1e-6). bq: float quadric as the
 * reference forms it; bq64: the same quadric formed in double (FP64 oracle only). */
static int boundary_prepare(const float v0[3], const float v1[3], const float vs[3], float bq[10], double bq64[10],
                            dda_state *st)
{
    double dir[3] = {(double)(v1[0] - v0[0]), (double)(v1[1] - v0[1]), (double)(v1[2] - v0[2])};
    const double sq = (dir[0] * dir[0] + dir[1] * dir[1]) + dir[2] * dir[2];
    const double len = sqrt(sq);
    if (len < 1e-6)
        return 0;
    if (sq > 0.0)
    {
        const double r = sqrt(sq);
        dir[0] /= r;
        dir[1] /= r;
        dir[2] /= r;
    }
    float A[9];
    double A64[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
        {
            const double o = dir[i] * dir[j];
            A[i * 3 + j] = (i == j ? 1.0f : 0.0f) - (float)o;
            A64[i * 3 + j] = (i == j ? 1.0 : 0.0) - o;
        }
    float b[3];
    double b64[3];
    for (int i = 0; i < 3; ++i)
    {
        b[i] = -dot3f(A[i * 3 + 0], A[i * 3 + 1], A[i * 3 + 2], v0[0], v0[1], v0[2]);
        b64[i] = -(A64[i * 3 + 0] * v0[0] + (A64[i * 3 + 1] * v0[1] + A64[i * 3 + 2] * v0[2]));
    }
    float r[3];
    double r64[3];
    for (int j = 0; j < 3; ++j)
    {
        r[j] = dot3f(v0[0], v0[1], v0[2], A[0 * 3 + j], A[1 * 3 + j], A[2 * 3 + j]);
        r64[j] = v0[0] * A64[0 * 3 + j] + (v0[1] * A64[1 * 3 + j] + v0[2] * A64[2 * 3 + j]);
    }
    const float c = dot3f(r[0], r[1], r[2], v0[0], v0[1], v0[2]);
    const double c64 = r64[0] * v0[0] + (r64[1] * v0[1] + r64[2] * v0[2]);
    bq[0] = A[0]; bq[1] = A[1]; bq[2] = A[2]; bq[3] = b[0];
    bq[4] = A[4]; bq[5] = A[5]; bq[6] = b[1];
    bq[7] = A[8]; bq[8] = b[2];
    bq[9] = c;
    bq64[0] = A64[0]; bq64[1] = A64[1]; bq64[2] = A64[2]; bq64[3] = b64[0];
    bq64[4] = A64[4]; bq64[5] = A64[5]; bq64[6] = b64[1];
    bq64[7] = A64[8]; bq64[8] = b64[2];
    bq64[9] = c64;

    int64_t span = 0;
    for (int a = 0; a < 3; ++a)
    {
        const int c0 = trunc_f2i(floorf(v0[a] / vs[a]));
        const int c1 = trunc_f2i(floorf(v1[a] / vs[a]));
        st->cur[a] = c0;
        st->step[a] = (dir[a] > 0) ? 1 : -1;
        if (dir[a] == 0.0)
        {
            st->tmax[a] = INFINITY;
            st->tdelta[a] = INFINITY;
        }
        else
        {
            const float border = vs[a] * (float)(c0 + (st->step[a] > 0 ? 1 : 0));
            st->tmax[a] = (double)(border - v0[a]) / dir[a];
            st->tdelta[a] = (double)vs[a] / fabs(dir[a]);
        }
        span += llabs((long long)c1 - (long long)c0) + 2;
    }
    st->len = len;
    st->started = 0;
    st->guard = span + 8;
    return 1;
}

/* Yields the start voxel, then one voxel per DDA step (flexible_dual_grid.cpp:481-507). */
static int dda_next(dda_state *st, int32_t out[3])
{
    if (!st->started)
    {
        st->started = 1;
        memcpy(out, st->cur, sizeof(st->cur));
        return 1;
    }
    int axis;
    if (st->tmax[0] < st->tmax[1])
        axis = (st->tmax[0] < st->tmax[2]) ? 0 : 2;
    else
        axis = (st->tmax[1] < st->tmax[2]) ? 1 : 2;
    if (st->tmax[axis] > st->len)
        return 0;
    if (--st->guard < 0)
        return 0; /* unreachable for finite input; keeps NaN input from looping */
    st->cur[axis] += st->step[axis];
    st->tmax[axis] += st->tdelta[axis];
    memcpy(out, st->cur, sizeof(st->cur));
    return 1;
}

/* ---------------- instantiate float and double bodies ---------------- */
#define REAL float
#define REAL_IS_FLOAT 1
#define REAL_EPS FLT_EPSILON
#define REAL_MIN FLT_MIN
#define REAL_SQRT sqrtf
#define REAL_ABS fabsf
#define FN(x) x##_f32
#include "fdg_oracle_impl.h"
#undef REAL
#undef REAL_IS_FLOAT
#undef REAL_EPS
#undef REAL_MIN
#undef REAL_SQRT
#undef REAL_ABS
#undef FN

#define REAL double
#define REAL_IS_FLOAT 0
#define REAL_EPS DBL_EPSILON
#define REAL_MIN DBL_MIN
#define REAL_SQRT sqrt
#define REAL_ABS fabs
#define FN(x) x##_f64
#include "fdg_oracle_impl.h"

/* ---------------- occupancy only (flexible_dual_grid.cpp:80-156) ---------------- */
typedef struct occ_acc
{
    vox_map map;
    int64_t n, cap;
    int32_t *vox;
    int oom;
} occ_acc;

static void occ_event(void *ctx, const int32_t c[3], int ax2, int dx, int dy, const double pt[3])
{
    (void)ax2; (void)dx; (void)dy; (void)pt;
    occ_acc *a = (occ_acc *)ctx;
    if (a->oom)
        return;
    const uint64_t key = map_key(c);
    if (map_find(&a->map, key) >= 0)
        return;
    if (a->n == a->cap)
    {
        a->cap = a->cap ? a->cap * 2 : 1024;
        a->vox = (int32_t *)realloc(a->vox, (size_t)a->cap * 3 * sizeof(int32_t));
        if (!a->vox)
        {
            a->oom = 1;
            return;
        }
    }
    if (map_insert(&a->map, key, a->n) != 0)
    {
        a->oom = 1;
        return;
    }
    memcpy(a->vox + a->n * 3, c, 3 * sizeof(int32_t));
    a->n++;
}

/* triangles: [T,3,3] float, grid-local coordinates. */
int fdg_oracle_intersect_occ(const float *tris, int64_t nt, const float vs[3], const int32_t grid_range[6],
                             int64_t *n_out, int32_t **vox_out)
{
    const int32_t gmin[3] = {grid_range[0], grid_range[1], grid_range[2]};
    const int32_t gmax[3] = {grid_range[3], grid_range[4], grid_range[5]};
    map_set_grid(gmin, gmax);
    occ_acc a;
    memset(&a, 0, sizeof(a));
    if (map_init(&a.map, 1 << 12) != 0)
        return FDG_ORACLE_OOM;
    for (int64_t t = 0; t < nt && !a.oom; ++t)
    {
        float v[3][3];
        memcpy(v, tris + t * 9, sizeof(v));
        scan_triangle(v, vs, gmin, gmax, occ_event, &a);
    }
    map_free(&a.map);
    if (a.oom)
    {
        free(a.vox);
        return FDG_ORACLE_OOM;
    }
    *n_out = a.n;
    *vox_out = a.vox;
    return 0;
}

void fdg_oracle_free(fdg_oracle_out *o)
{
    free(o->voxels);
    free(o->dual);
    free(o->intersected);
    free(o->qef);
    free(o->mean_sum);
    free(o->cnt);
    memset(o, 0, sizeof(*o));
}

void fdg_oracle_free_ptr(void *p)
{
    free(p);
}

/*
 * z-order codes of o_voxel.serialize.encode_seq / decode_seq, mode 'z_order'
 * (serialize/z_order.cu:33-97 and serialize.py:7-36): bit i of x, y and z goes
 * to bits 3i+2, 3i+1 and 3i of a 30-bit code (x the most significant of each
 * triple), for coordinates in [0, 1024).
 */
void fdg_oracle_z_order_encode(int64_t n, const int32_t *x, const int32_t *y, const int32_t *z, int32_t *codes)
{
    for (int64_t k = 0; k < n; ++k)
    {
        uint32_t c = 0;
        for (int i = 0; i < 10; ++i)
        {
            c |= (((uint32_t)x[k] >> i) & 1u) << (3 * i + 2);
            c |= (((uint32_t)y[k] >> i) & 1u) << (3 * i + 1);
            c |= (((uint32_t)z[k] >> i) & 1u) << (3 * i);
        }
        codes[k] = (int32_t)c;
    }
}

void fdg_oracle_z_order_decode(int64_t n, const int32_t *codes, int32_t *x, int32_t *y, int32_t *z)
{
    for (int64_t k = 0; k < n; ++k)
    {
        const uint32_t c = (uint32_t)codes[k];
        uint32_t a = 0, b = 0, d = 0;
        for (int i = 0; i < 10; ++i)
        {
            a |= ((c >> (3 * i + 2)) & 1u) << i;
            b |= ((c >> (3 * i + 1)) & 1u) << i;
            d |= ((c >> (3 * i)) & 1u) << i;
        }
        x[k] = (int32_t)a;
        y[k] = (int32_t)b;
        z[k] = (int32_t)d;
    }
}

/*
 * Hilbert codes of o_voxel.serialize.encode_seq / decode_seq, mode 'hilbert'
 * (serialize/hilbert.cu:33-130 and serialize.py:7-66).  The reference uses
 * J. Skilling's transposed-index form of the Hilbert curve ("Programming the
 * Hilbert curve", AIP Conf. Proc. 707, 2004) for 3 axes of 10 bits: the axes
 * are turned into the transposed index (undo the excess work bit plane by bit
 * plane from the top, then Gray-encode), and the three transposed words are
 * interleaved like the z-order code (word 0 the most significant of each
 * triple).  Decoding runs the inverse steps.  Coordinates in [0, 1024).
 */
static void skilling_axes_to_transpose(uint32_t a[3])
{
    for (uint32_t q = 1u << 9; q > 1u; q >>= 1)
    {
        const uint32_t low = q - 1u;
        for (int i = 0; i < 3; ++i)
        {
            if (a[i] & q)
                a[0] ^= low;
            else
            {
                const uint32_t swap = (a[0] ^ a[i]) & low;
                a[0] ^= swap;
                a[i] ^= swap;
            }
        }
    }
    a[1] ^= a[0];
    a[2] ^= a[1];
    uint32_t flip = 0;
    for (uint32_t q = 1u << 9; q > 1u; q >>= 1)
        if (a[2] & q)
            flip ^= q - 1u;
    a[0] ^= flip;
    a[1] ^= flip;
    a[2] ^= flip;
}

static void skilling_transpose_to_axes(uint32_t a[3])
{
    const uint32_t half = a[2] >> 1;
    a[2] ^= a[1];
    a[1] ^= a[0];
    a[0] ^= half;
    for (uint32_t q = 2u; q != (1u << 10); q <<= 1)
    {
        const uint32_t low = q - 1u;
        for (int i = 2; i >= 0; --i)
        {
            if (a[i] & q)
                a[0] ^= low;
            else
            {
                const uint32_t swap = (a[0] ^ a[i]) & low;
                a[0] ^= swap;
                a[i] ^= swap;
            }
        }
    }
}

void fdg_oracle_hilbert_encode(int64_t n, const int32_t *x, const int32_t *y, const int32_t *z, int32_t *codes)
{
    for (int64_t k = 0; k < n; ++k)
    {
        uint32_t a[3] = {(uint32_t)x[k] & 1023u, (uint32_t)y[k] & 1023u, (uint32_t)z[k] & 1023u};
        skilling_axes_to_transpose(a);
        uint32_t c = 0;
        for (int i = 0; i < 10; ++i)
        {
            c |= ((a[0] >> i) & 1u) << (3 * i + 2);
            c |= ((a[1] >> i) & 1u) << (3 * i + 1);
            c |= ((a[2] >> i) & 1u) << (3 * i);
        }
        codes[k] = (int32_t)c;
    }
}

void fdg_oracle_hilbert_decode(int64_t n, const int32_t *codes, int32_t *x, int32_t *y, int32_t *z)
{
    for (int64_t k = 0; k < n; ++k)
    {
        const uint32_t c = (uint32_t)codes[k];
        uint32_t a[3] = {0, 0, 0};
        for (int i = 0; i < 10; ++i)
        {
            a[0] |= ((c >> (3 * i + 2)) & 1u) << i;
            a[1] |= ((c >> (3 * i + 1)) & 1u) << i;
            a[2] |= ((c >> (3 * i)) & 1u) << i;
        }
        skilling_transpose_to_axes(a);
        x[k] = (int32_t)a[0];
        y[k] = (int32_t)a[1];
        z[k] = (int32_t)a[2];
    }
}
