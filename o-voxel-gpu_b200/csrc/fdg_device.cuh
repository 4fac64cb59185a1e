// fdg_device.cuh -- device-side geometry for mesh -> flexible dual grid.
//
// Every floating-point expression here reproduces the reference CPU path
// (src/convert/flexible_dual_grid.cpp) operation by operation.  The
// translation unit is compiled with -fmad=false, so no multiply-add pair is
// contracted into an FMA (the x86-64 reference build has none either), and
// with IEEE division and square root (nvcc defaults, no fast math).  Fixed
// reduction orders (the reference uses Eigen fixed-size objects):
//   3 floats  a0*b0 + (a1*b1 + a2*b2)
//   4 floats  (a0*b0 + a2*b2) + (a1*b1 + a3*b3)
//   3 doubles (a0*b0 + a1*b1) + a2*b2
//   runtime-sized reductions left to right.
#pragma once

#include <cstdint>
#include <climits>
#include <cfloat>

namespace ovx
{

// Voxels are stored in 8x8x8 bricks; one brick = 16 x 32-bit words of
// occupancy.  Word w = lz*2 + (ly>>2), bit b = (ly&3)*8 + lx, so the bit
// index inside a brick is lx + 8*ly + 64*lz.
constexpr int kBrick = 8;
constexpr int kWordsPerBrick = 16;

struct Grid
{
    float vs[3];
    int gmin[3];
    int gmax[3];
    int size[3];  // gmax - gmin
    int nb[3];    // bricks per axis
    long long nbricks;
    double rv[3]; // 1 / (double)vs, for trunc_div
};

// ---- x86 conversion semantics: out-of-range and NaN give INT_MIN ----
__device__ __forceinline__ int trunc_d2i(double d)
{
    return (d > -2147483649.0 && d < 2147483648.0) ? (int)d : INT_MIN;
}
__device__ __forceinline__ int trunc_f2i(float f)
{
    return (f > -2147483904.0f && f < 2147483648.0f) ? (int)f : INT_MIN;
}
__device__ __forceinline__ int clampi(int v, int lo, int hi)
{
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

// trunc_d2i(a / b) with the IEEE quotient, computed from q = a * rb
// (rb = 1/b) when that is provably equivalent.  |q - a/b| and |RN(a/b) - a/b|
// are both below 2.3e-16 |a/b|, so if q's fractional part keeps 1e-12|q| away
// from an integer, RN(a/b) lies in the same open unit interval and truncates
// to the same integer.  Otherwise (near an integer, near zero, out of int
// range, NaN) the exact division decides.
__device__ __forceinline__ int trunc_div(double a, double b, double rb)
{
    const double q = a * rb;
    const double aq = fabs(q);
    if (aq < 2.0e9)
    {
        const double fl = floor(q);
        const double fr = q - fl;
        const double d = 1e-12 * (aq > 1.0 ? aq : 1.0);
        if (fr > d && fr < 1.0 - d)
            return (int)(q >= 0.0 ? fl : fl + 1.0);
    }
    return trunc_d2i(a / b);
}
__device__ __forceinline__ float dot3f(float a0, float a1, float a2, float b0, float b1, float b2)
{
    return a0 * b0 + (a1 * b1 + a2 * b2);
}
__device__ __forceinline__ float dot2f(float a0, float a1, float b0, float b1)
{
    return a0 * b0 + a1 * b1;
}
__device__ __forceinline__ float dot4v(const float a[4], const float b[4])
{
    return (a[0] * b[0] + a[2] * b[2]) + (a[1] * b[1] + a[3] * b[3]);
}
__device__ __forceinline__ float max0f(float a)
{
    return (a < 0.0f) ? 0.0f : a;
}

// ---- brick addressing ----
__device__ __forceinline__ bool in_grid(const Grid &g, int x, int y, int z)
{
    return x >= g.gmin[0] && x < g.gmax[0] && y >= g.gmin[1] && y < g.gmax[1] && z >= g.gmin[2] && z < g.gmax[2];
}
// word index and bit of an in-grid voxel
__device__ __forceinline__ long long voxel_word(const Grid &g, int x, int y, int z, uint32_t &bit)
{
    const int rx = x - g.gmin[0], ry = y - g.gmin[1], rz = z - g.gmin[2];
    const long long b = (long long)(rx >> 3) + (long long)g.nb[0] * ((long long)(ry >> 3) + (long long)g.nb[1] * (long long)(rz >> 3));
    bit = ((uint32_t)(ry & 3) << 3) | (uint32_t)(rx & 7);
    return b * kWordsPerBrick + ((rz & 7) << 1) + ((ry & 7) >> 2);
}

// ---- triangle load: vertices shifted into grid-local coordinates in float ----
template <typename IndexT>
__device__ __forceinline__ bool load_triangle(const float *__restrict__ verts, long long nv, const IndexT *__restrict__ faces,
                                              long long t, const float origin[3], float v[3][3], long long idx[3])
{
    bool ok = true;
    for (int k = 0; k < 3; ++k)
    {
        long long i = faces ? (long long)faces[t * 3 + k] : t * 3 + k;
        idx[k] = i;
        if (i < 0 || i >= nv)
        {
            ok = false;
            i = 0;
        }
        v[k][0] = verts[i * 3 + 0] - origin[0];
        v[k][1] = verts[i * 3 + 1] - origin[1];
        v[k][2] = verts[i * 3 + 2] - origin[2];
    }
    return ok;
}

// normalize(cross(v1 - v0, v2 - v1)) with Eigen normalized() semantics
__device__ __forceinline__ void tri_normal(const float v[3][3], float n[3])
{
    const float e0x = v[1][0] - v[0][0], e0y = v[1][1] - v[0][1], e0z = v[1][2] - v[0][2];
    const float e1x = v[2][0] - v[1][0], e1y = v[2][1] - v[1][1], e1z = v[2][2] - v[1][2];
    n[0] = e0y * e1z - e0z * e1y;
    n[1] = e0z * e1x - e0x * e1z;
    n[2] = e0x * e1y - e0y * e1x;
    const float s = dot3f(n[0], n[1], n[2], n[0], n[1], n[2]);
    if (s > 0.0f)
    {
        const float r = sqrtf(s);
        n[0] = n[0] / r;
        n[1] = n[1] / r;
        n[2] = n[2] / r;
    }
}

// plane quadric plane*plane^T, plane = (n, -n.v0); 10 upper entries
__device__ __forceinline__ void tri_quadric(const float v[3][3], float q[10])
{
    float n[3];
    tri_normal(v, n);
    const float d = -dot3f(n[0], n[1], n[2], v[0][0], v[0][1], v[0][2]);
    q[0] = n[0] * n[0];
    q[1] = n[0] * n[1];
    q[2] = n[0] * n[2];
    q[3] = n[0] * d;
    q[4] = n[1] * n[1];
    q[5] = n[1] * n[2];
    q[6] = n[1] * d;
    q[7] = n[2] * n[2];
    q[8] = n[2] * d;
    q[9] = d * d;
}

// ---------------------------------------------------------------------------
// Scanline setup for one projection axis (flexible_dual_grid.cpp:195-211)
// ---------------------------------------------------------------------------
struct AxisScan
{
    double t[3][3]; // rows sorted by y; components (x=ax0, y=ax1, z=ax2)
    int start, mid, end;
    int ax0, ax1, ax2;
};

__device__ __forceinline__ void axis_setup(const float v[3][3], int ax2, const Grid &g, AxisScan &s)
{
    s.ax2 = ax2;
    s.ax0 = (ax2 + 1) % 3;
    s.ax1 = (ax2 + 2) % 3;
    double t[3][3];
    for (int k = 0; k < 3; ++k)
    {
        t[k][0] = (double)v[k][s.ax0];
        t[k][1] = (double)v[k][s.ax1];
        t[k][2] = (double)v[k][s.ax2];
    }
    // stable insertion sort by y (libstdc++ std::sort on three elements)
    for (int i = 1; i < 3; ++i)
    {
        const double a = t[i][0], b = t[i][1], c = t[i][2];
        int j = i;
        while (j > 0 && b < t[j - 1][1])
        {
            t[j][0] = t[j - 1][0];
            t[j][1] = t[j - 1][1];
            t[j][2] = t[j - 1][2];
            --j;
        }
        t[j][0] = a;
        t[j][1] = b;
        t[j][2] = c;
    }
    for (int k = 0; k < 3; ++k)
        for (int c = 0; c < 3; ++c)
            s.t[k][c] = t[k][c];
    const double vy = (double)g.vs[s.ax1];
    const double ry = g.rv[s.ax1];
    const int lo = g.gmin[s.ax1], hi = g.gmax[s.ax1] - 1;
    s.start = clampi(trunc_div(t[0][1], vy, ry), lo, hi);
    s.mid = clampi(trunc_div(t[1][1], vy, ry), lo, hi);
    s.end = clampi(trunc_div(t[2][1], vy, ry), lo, hi);
}

// Column bound of the projected triangle on ax0 (for work estimates and tiling):
// [clo, chi] with clo/chi the clamped truncated extremes.
__device__ __forceinline__ void axis_col_bounds(const AxisScan &s, const Grid &g, int &clo, int &chi)
{
    double mn = s.t[0][0], mx = s.t[0][0];
    for (int k = 1; k < 3; ++k)
    {
        mn = s.t[k][0] < mn ? s.t[k][0] : mn;
        mx = s.t[k][0] > mx ? s.t[k][0] : mx;
    }
    const double vx = (double)g.vs[s.ax0];
    const double rx = g.rv[s.ax0];
    clo = clampi(trunc_div(mn, vx, rx), g.gmin[s.ax0], g.gmax[s.ax0] - 1);
    chi = clampi(trunc_div(mx, vx, rx), g.gmin[s.ax0], g.gmax[s.ax0] - 1);
}

// Events of one scan row, columns restricted to [col_lo, col_hi).
// emit(xi, yi, zi, x_float, y_float, z_double) in (ax0, ax1, ax2) order.
// One scanline row yi of a projection axis (flexible_dual_grid.cpp:219-236):
// the two edge crossings (t3, t4), sorted along x, and the column range.
struct RowSetup
{
    double t3x, t3z, t4x, t4z;
    int x0, x1; // columns xi in [x0, x1)
};

__device__ __forceinline__ void row_setup(const AxisScan &s, int yi, int col_lo, int col_hi, const Grid &g, RowSetup &r)
{
    const bool first = yi < s.mid;
    const double *T0 = first ? s.t[0] : s.t[2];
    const double *T1 = s.t[1];
    const double *T2 = first ? s.t[2] : s.t[0];
    const float yf = (float)(yi + 1) * g.vs[s.ax1];
    const double y = (double)yf;
    double t3x, t3z, t4x, t4z;
    if (T0[1] == T1[1])
    {
        t3x = T0[0];
        t3z = T0[2];
    }
    else
    {
        const double al = (y - T0[1]) / (T1[1] - T0[1]);
        const double om = 1.0 - al;
        t3x = om * T0[0] + al * T1[0];
        t3z = om * T0[2] + al * T1[2];
    }
    if (T0[1] == T2[1])
    {
        t4x = T0[0];
        t4z = T0[2];
    }
    else
    {
        const double al = (y - T0[1]) / (T2[1] - T0[1]);
        const double om = 1.0 - al;
        t4x = om * T0[0] + al * T2[0];
        t4z = om * T0[2] + al * T2[2];
    }
    if (t3x > t4x)
    {
        double tmp = t3x;
        t3x = t4x;
        t4x = tmp;
        tmp = t3z;
        t3z = t4z;
        t4z = tmp;
    }
    const double vx = (double)g.vs[s.ax0];
    const double rx = g.rv[s.ax0];
    const int ls = clampi(trunc_div(t3x, vx, rx), g.gmin[s.ax0], g.gmax[s.ax0] - 1);
    const int le = clampi(trunc_div(t4x, vx, rx), g.gmin[s.ax0], g.gmax[s.ax0] - 1);
    r.t3x = t3x;
    r.t3z = t3z;
    r.t4x = t4x;
    r.t4z = t4z;
    r.x0 = ls > col_lo ? ls : col_lo;
    r.x1 = le < col_hi ? le : col_hi;
}

// Crossing of column xi with a row (flexible_dual_grid.cpp:238-250): its z and
// voxel index zi along the projection axis.
__device__ __forceinline__ void col_event(const RowSetup &r, int xi, int ax0, int ax2, const Grid &g, double &z, int &zi)
{
    const float xf = (float)(xi + 1) * g.vs[ax0];
    const double x = (double)xf;
    if (r.t3x == r.t4x)
        z = r.t3z;
    else
    {
        const double al = (x - r.t3x) / (r.t4x - r.t3x);
        z = (1.0 - al) * r.t3z + al * r.t4z;
    }
    zi = trunc_div(z, (double)g.vs[ax2], g.rv[ax2]);
}

template <typename Emit>
__device__ __forceinline__ void scan_row(const AxisScan &s, int yi, int col_lo, int col_hi, const Grid &g, Emit &emit)
{
    RowSetup r;
    row_setup(s, yi, col_lo, col_hi, g, r);
    const float yf = (float)(yi + 1) * g.vs[s.ax1];
    for (int xi = r.x0; xi < r.x1; ++xi)
    {
        double z;
        int zi;
        col_event(r, xi, s.ax0, s.ax2, g, z, zi);
        if (zi >= g.gmin[s.ax2] && zi < g.gmax[s.ax2])
            emit(xi, yi, zi, (float)(xi + 1) * g.vs[s.ax0], yf, z);
    }
}

// ---------------------------------------------------------------------------
// Face stage: triangle / voxel-box overlap predicates (flexible_dual_grid.cpp:304-402)
// ---------------------------------------------------------------------------
struct FaceSetup
{
    float n[3];
    float d1, d2;
    float nxy[3][2], dxy[3];
    float nyz[3][2], dyz[3];
    float nzx[3][2], dzx[3];
    int bmin[3], bmax[3];
};

// Face-test voxel box [bmin, bmax) of a triangle (flexible_dual_grid.cpp:314-322).
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

__device__ __forceinline__ void face_setup(const float v[3][3], const Grid &g, FaceSetup &fs)
{
    float e[3][3];
    for (int c = 0; c < 3; ++c)
    {
        e[0][c] = v[1][c] - v[0][c];
        e[1][c] = v[2][c] - v[1][c];
        e[2][c] = v[0][c] - v[2][c];
    }
    tri_normal(v, fs.n);
    const float *n = fs.n;
    face_box(v, g, fs.bmin, fs.bmax);
    const float c0 = n[0] > 0.0f ? g.vs[0] : 0.0f;
    const float c1 = n[1] > 0.0f ? g.vs[1] : 0.0f;
    const float c2 = n[2] > 0.0f ? g.vs[2] : 0.0f;
    fs.d1 = dot3f(n[0], n[1], n[2], c0 - v[0][0], c1 - v[0][1], c2 - v[0][2]);
    fs.d2 = dot3f(n[0], n[1], n[2], (g.vs[0] - c0) - v[0][0], (g.vs[1] - c1) - v[0][1], (g.vs[2] - c2) - v[0][2]);
    const float mxy = (n[2] < 0.0f) ? -1.0f : 1.0f;
    const float myz = (n[0] < 0.0f) ? -1.0f : 1.0f;
    const float mzx = (n[1] < 0.0f) ? -1.0f : 1.0f;
    for (int k = 0; k < 3; ++k)
    {
        fs.nxy[k][0] = (-mxy) * e[k][1];
        fs.nxy[k][1] = mxy * e[k][0];
        fs.dxy[k] = -dot2f(fs.nxy[k][0], fs.nxy[k][1], v[k][0], v[k][1]) +
                    dot2f(max0f(fs.nxy[k][0]), max0f(fs.nxy[k][1]), g.vs[0], g.vs[1]);
        fs.nyz[k][0] = (-myz) * e[k][2];
        fs.nyz[k][1] = myz * e[k][1];
        fs.dyz[k] = -dot2f(fs.nyz[k][0], fs.nyz[k][1], v[k][1], v[k][2]) +
                    dot2f(max0f(fs.nyz[k][0]), max0f(fs.nyz[k][1]), g.vs[1], g.vs[2]);
        fs.nzx[k][0] = (-mzx) * e[k][0];
        fs.nzx[k][1] = mzx * e[k][2];
        fs.dzx[k] = -dot2f(fs.nzx[k][0], fs.nzx[k][1], v[k][2], v[k][0]) +
                    dot2f(max0f(fs.nzx[k][0]), max0f(fs.nzx[k][1]), g.vs[2], g.vs[0]);
    }
}

// Face-test coefficients by index: 0-2 n, 3 d1, 4 d2, 5-10 nxy[k][c] (k*2+c),
// 11-13 dxy, 14-19 nyz, 20-22 dyz, 23-28 nzx, 29-31 dzx.
constexpr int kFaceCoef = 32;

__device__ __forceinline__ void face_coefs(const FaceSetup &fs, float c[kFaceCoef])
{
    c[0] = fs.n[0];
    c[1] = fs.n[1];
    c[2] = fs.n[2];
    c[3] = fs.d1;
    c[4] = fs.d2;
#pragma unroll
    for (int k = 0; k < 3; ++k)
    {
        c[5 + 2 * k] = fs.nxy[k][0];
        c[6 + 2 * k] = fs.nxy[k][1];
        c[11 + k] = fs.dxy[k];
        c[14 + 2 * k] = fs.nyz[k][0];
        c[15 + 2 * k] = fs.nyz[k][1];
        c[20 + k] = fs.dyz[k];
        c[23 + 2 * k] = fs.nzx[k][0];
        c[24 + 2 * k] = fs.nzx[k][1];
        c[29 + k] = fs.dzx[k];
    }
}

// Box-triangle test at the voxel's min corner (flexible_dual_grid.cpp:324-409):
// plane slab and the 9 projected edge half-planes.  All ten are evaluated and
// combined (the reference stops at the first failing one; the result is the
// same), so the lanes of a warp do not diverge on where they stop.  `C(i)`
// returns face-test coefficient i (see kFaceCoef), so registers and shared
// memory share one code path.
template <typename Coef>
__device__ __forceinline__ bool face_test_c(const Coef &C, const Grid &g, int x, int y, int z)
{
    const float p0 = g.vs[0] * (float)x, p1 = g.vs[1] * (float)y, p2 = g.vs[2] * (float)z;
    const float nd = dot3f(C(0), C(1), C(2), p0, p1, p2);
    bool ok = !((nd + C(3)) * (nd + C(4)) > 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        ok &= !(dot2f(C(5 + 2 * k), C(6 + 2 * k), p0, p1) + C(11 + k) < 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        ok &= !(dot2f(C(14 + 2 * k), C(15 + 2 * k), p1, p2) + C(20 + k) < 0.0f);
#pragma unroll
    for (int k = 0; k < 3; ++k)
        ok &= !(dot2f(C(23 + 2 * k), C(24 + 2 * k), p2, p0) + C(29 + k) < 0.0f);
    return ok;
}

// True when no voxel of the index box [lo, hi) (absolute voxel indices, each
// range non-empty) can pass face_test_c.  Exact, not an estimate: every test
// is a sum of products of a fixed coefficient and a coordinate vs * i, and
// IEEE rounding is monotone, so each computed test value is monotone in every
// coordinate; evaluated with the same operations at the box corner that
// maximises (or minimises) it, it bounds the computed value of every voxel of
// the box.  A test that fails at its best corner fails for the whole box.
// NaN coefficients reject nothing (every comparison is false).
template <typename Coef>
__device__ __forceinline__ bool face_box_rejects(const Coef &C, const Grid &g, const int lo[3], const int hi[3])
{
    // coordinate of axis a at the corner maximising (want_max) or minimising c * p
    auto pick = [&](float c, int a, bool want_max) -> float {
        const int i = ((c >= 0.0f) == want_max) ? hi[a] - 1 : lo[a];
        return g.vs[a] * (float)i;
    };
    // plane slab: fails where (nd + d1) and (nd + d2) are both positive (or
    // both negative) with a positive product; nd is smallest (largest) at one corner
    const float nlo = dot3f(C(0), C(1), C(2), pick(C(0), 0, false), pick(C(1), 1, false), pick(C(2), 2, false));
    const float ul = nlo + C(3), wl = nlo + C(4);
    if (ul > 0.0f && wl > 0.0f && ul * wl > 0.0f)
        return true;
    const float nhi = dot3f(C(0), C(1), C(2), pick(C(0), 0, true), pick(C(1), 1, true), pick(C(2), 2, true));
    const float uh = nhi + C(3), wh = nhi + C(4);
    if (uh < 0.0f && wh < 0.0f && uh * wh > 0.0f)
        return true;
    // the 9 edge half-planes: fail where the value is negative; largest at one corner
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (dot2f(C(5 + 2 * k), C(6 + 2 * k), pick(C(5 + 2 * k), 0, true), pick(C(6 + 2 * k), 1, true)) + C(11 + k) < 0.0f)
            return true;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (dot2f(C(14 + 2 * k), C(15 + 2 * k), pick(C(14 + 2 * k), 1, true), pick(C(15 + 2 * k), 2, true)) + C(20 + k) < 0.0f)
            return true;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (dot2f(C(23 + 2 * k), C(24 + 2 * k), pick(C(23 + 2 * k), 2, true), pick(C(24 + 2 * k), 0, true)) + C(29 + k) < 0.0f)
            return true;
    return false;
}

struct FaceCoefRegs
{
    const FaceSetup &fs;
    __device__ __forceinline__ float operator()(int i) const
    {
        switch (i)
        {
        case 0: return fs.n[0];
        case 1: return fs.n[1];
        case 2: return fs.n[2];
        case 3: return fs.d1;
        case 4: return fs.d2;
        default: break;
        }
        if (i < 11)
            return fs.nxy[(i - 5) >> 1][(i - 5) & 1];
        if (i < 14)
            return fs.dxy[i - 11];
        if (i < 20)
            return fs.nyz[(i - 14) >> 1][(i - 14) & 1];
        if (i < 23)
            return fs.dyz[i - 20];
        if (i < 29)
            return fs.nzx[(i - 23) >> 1][(i - 23) & 1];
        return fs.dzx[i - 29];
    }
};

__device__ __forceinline__ bool face_test(const FaceSetup &fs, const Grid &g, int x, int y, int z)
{
    return face_test_c(FaceCoefRegs{fs}, g, x, y, z);
}

// ---------------------------------------------------------------------------
// Boundary stage: line quadric and 3D DDA (flexible_dual_grid.cpp:427-507)
// ---------------------------------------------------------------------------
struct Dda
{
    int cur[3];
    int step[3];
    double tmax[3], tdelta[3];
    double len;
    int guard;
};

// Returns false for segments shorter than 1e-6 (skipped by the reference).
// q (optional) receives the unweighted line quadric, 10 upper entries.
__device__ __forceinline__ bool boundary_setup(const float v0[3], const float v1[3], const Grid &g, Dda &d, float *q)
{
    double dir[3] = {(double)(v1[0] - v0[0]), (double)(v1[1] - v0[1]), (double)(v1[2] - v0[2])};
    const double sq = (dir[0] * dir[0] + dir[1] * dir[1]) + dir[2] * dir[2];
    const double len = sqrt(sq);
    if (len < 1e-6)
        return false;
    if (sq > 0.0)
    {
        const double r = sqrt(sq);
        dir[0] = dir[0] / r;
        dir[1] = dir[1] / r;
        dir[2] = dir[2] / r;
    }
    if (q)
    {
        float A[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                A[i * 3 + j] = (i == j ? 1.0f : 0.0f) - (float)(dir[i] * dir[j]);
        float b[3], r[3];
        for (int i = 0; i < 3; ++i)
            b[i] = -dot3f(A[i * 3 + 0], A[i * 3 + 1], A[i * 3 + 2], v0[0], v0[1], v0[2]);
        for (int j = 0; j < 3; ++j)
            r[j] = dot3f(v0[0], v0[1], v0[2], A[0 * 3 + j], A[1 * 3 + j], A[2 * 3 + j]);
        const float c = dot3f(r[0], r[1], r[2], v0[0], v0[1], v0[2]);
        q[0] = A[0];
        q[1] = A[1];
        q[2] = A[2];
        q[3] = b[0];
        q[4] = A[4];
        q[5] = A[5];
        q[6] = b[1];
        q[7] = A[8];
        q[8] = b[2];
        q[9] = c;
    }
    int span = 0;
    for (int a = 0; a < 3; ++a)
    {
        const int c0 = trunc_f2i(floorf(v0[a] / g.vs[a]));
        const int c1 = trunc_f2i(floorf(v1[a] / g.vs[a]));
        d.cur[a] = c0;
        d.step[a] = (dir[a] > 0) ? 1 : -1;
        if (dir[a] == 0.0)
        {
            d.tmax[a] = __longlong_as_double(0x7ff0000000000000LL);
            d.tdelta[a] = __longlong_as_double(0x7ff0000000000000LL);
        }
        else
        {
            const float border = g.vs[a] * (float)(c0 + (d.step[a] > 0 ? 1 : 0));
            d.tmax[a] = (double)(border - v0[a]) / dir[a];
            d.tdelta[a] = (double)g.vs[a] / fabs(dir[a]);
        }
        long long df = (long long)c1 - (long long)c0;
        df = df < 0 ? -df : df;
        span += (int)(df > (1 << 28) ? (1 << 28) : df) + 2;
    }
    d.len = len;
    d.guard = span + 8;
    return true;
}

// Advance to the next voxel; false when the walk passed the segment end (or the step guard ran out).
__device__ __forceinline__ bool dda_step(Dda &d)
{
    int axis;
    if (d.tmax[0] < d.tmax[1])
        axis = (d.tmax[0] < d.tmax[2]) ? 0 : 2;
    else
        axis = (d.tmax[1] < d.tmax[2]) ? 1 : 2;
    if (d.tmax[axis] > d.len)
        return false;
    if (--d.guard < 0)
        return false;
    d.cur[axis] += d.step[axis];
    d.tmax[axis] += d.tdelta[axis];
    return true;
}

// ---------------------------------------------------------------------------
// Per-voxel solve (flexible_dual_grid.cpp:766-983)
// ---------------------------------------------------------------------------
// Column-pivoting Householder QR solve, A row-major n x n (n = 2 or 3).
// Scalar arithmetic of the solves: the float members are the exact path's
// operations (Eigen's fixed-size reduction orders), the double ones serve the
// compensated-precision mode.
template <typename T>
struct Arith;

template <>
struct Arith<float>
{
    static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
    static __device__ __forceinline__ float tiny() { return FLT_MIN; }
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float abs(float x) { return fabsf(x); }
    static __device__ __forceinline__ float dot3(float a0, float a1, float a2, float b0, float b1, float b2)
    {
        return dot3f(a0, a1, a2, b0, b1, b2);
    }
    static __device__ __forceinline__ float dot4(const float a[4], const float b[4]) { return dot4v(a, b); }
};

template <>
struct Arith<double>
{
    static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
    static __device__ __forceinline__ double tiny() { return DBL_MIN; }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double abs(double x) { return fabs(x); }
    static __device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1, double b2)
    {
        return (a0 * b0 + a1 * b1) + a2 * b2;
    }
    static __device__ __forceinline__ double dot4(const double a[4], const double b[4])
    {
        return ((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]) + a[3] * b[3];
    }
};

template <typename T, int N>
__device__ __forceinline__ void cpqr_solve_t(const T *A, const T *b, T *x, T *rdiag = nullptr)
{
    using Ar = Arith<T>;
    T qr[N * N], c[N], h[N], nu[N], nd[N];
    int perm[N];
#pragma unroll
    for (int i = 0; i < N * N; ++i)
        qr[i] = A[i];
#pragma unroll
    for (int i = 0; i < N; ++i)
    {
        c[i] = b[i];
        perm[i] = i;
        x[i] = T(0);
    }
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
        T s;
        if (N == 3)
            s = qr[0 * N + j] * qr[0 * N + j] + (qr[1 * N + j] * qr[1 * N + j] + qr[2 * N + j] * qr[2 * N + j]);
        else
            s = qr[0 * N + j] * qr[0 * N + j] + qr[1 * N + j] * qr[1 * N + j];
        nd[j] = nu[j] = Ar::sqrt(s);
    }
    T maxn = nu[0];
#pragma unroll
    for (int j = 1; j < N; ++j)
        if (nu[j] > maxn)
            maxn = nu[j];
    const T th = (maxn * Ar::eps()) * (maxn * Ar::eps()) / (T)N;
    const T downdate_th = Ar::sqrt(Ar::eps());
    int nz = N;
#pragma unroll
    for (int k = 0; k < N; ++k)
    {
        int bi = k;
        T bv = nu[k];
#pragma unroll
        for (int j = k + 1; j < N; ++j)
            if (nu[j] > bv)
            {
                bv = nu[j];
                bi = j;
            }
        if (nz == N && bv * bv < th * (T)(N - k))
            nz = k;
        if (bi != k)
        {
#pragma unroll
            for (int r = 0; r < N; ++r)
            {
                const T t = qr[r * N + k];
                // bi is data dependent; select instead of dynamic indexing keeps arrays in registers
#pragma unroll
                for (int j = k + 1; j < N; ++j)
                    if (j == bi)
                    {
                        qr[r * N + k] = qr[r * N + j];
                        qr[r * N + j] = t;
                    }
            }
#pragma unroll
            for (int j = k + 1; j < N; ++j)
                if (j == bi)
                {
                    T t = nu[k];
                    nu[k] = nu[j];
                    nu[j] = t;
                    t = nd[k];
                    nd[k] = nd[j];
                    nd[j] = t;
                    const int ti = perm[k];
                    perm[k] = perm[j];
                    perm[j] = ti;
                }
        }
        const int len = N - k - 1;
        const T c0 = qr[k * N + k];
        T tsq = T(0);
#pragma unroll
        for (int i = 0; i < len; ++i)
        {
            const T e = qr[(k + 1 + i) * N + k];
            tsq = (i == 0) ? e * e : tsq + e * e;
        }
        T tau, beta;
        if (tsq <= Ar::tiny())
        {
            tau = T(0);
            beta = c0;
#pragma unroll
            for (int i = 0; i < len; ++i)
                qr[(k + 1 + i) * N + k] = T(0);
        }
        else
        {
            beta = Ar::sqrt(c0 * c0 + tsq);
            if (c0 >= T(0))
                beta = -beta;
            const T den = c0 - beta;
#pragma unroll
            for (int i = 0; i < len; ++i)
                qr[(k + 1 + i) * N + k] = qr[(k + 1 + i) * N + k] / den;
            tau = (beta - c0) / beta;
        }
        qr[k * N + k] = beta;
        h[k] = tau;
        if (len > 0 && tau != T(0))
        {
#pragma unroll
            for (int j = k + 1; j < N; ++j)
            {
                T tmp = T(0);
#pragma unroll
                for (int i = 0; i < len; ++i)
                {
                    const T p = qr[(k + 1 + i) * N + k] * qr[(k + 1 + i) * N + j];
                    tmp = (i == 0) ? p : tmp + p;
                }
                tmp = tmp + qr[k * N + j];
                qr[k * N + j] = qr[k * N + j] - tau * tmp;
#pragma unroll
                for (int i = 0; i < len; ++i)
                    qr[(k + 1 + i) * N + j] = qr[(k + 1 + i) * N + j] - (tau * qr[(k + 1 + i) * N + k]) * tmp;
            }
        }
#pragma unroll
        for (int j = k + 1; j < N; ++j)
        {
            if (nu[j] != T(0))
            {
                T temp = Ar::abs(qr[k * N + j]) / nu[j];
                temp = (T(1) + temp) * (T(1) - temp);
                temp = temp < T(0) ? T(0) : temp;
                const T ratio = nu[j] / nd[j];
                const T temp2 = temp * (ratio * ratio);
                if (temp2 <= downdate_th)
                {
                    T s = T(0);
#pragma unroll
                    for (int r = k + 1; r < N; ++r)
                    {
                        const T e = qr[r * N + j];
                        s = (r == k + 1) ? e * e : s + e * e;
                    }
                    nd[j] = nu[j] = Ar::sqrt(s);
                }
                else
                {
                    nu[j] = nu[j] * Ar::sqrt(temp);
                }
            }
        }
    }
    if (rdiag)
    {
#pragma unroll
        for (int k = 0; k < N; ++k)
            rdiag[k] = qr[k * N + k];
    }
    if (nz == 0)
        return;
#pragma unroll
    for (int k = 0; k < N; ++k)
    {
        if (k >= nz)
            break;
        const int len = N - k - 1;
        const T tau = h[k];
        if (len == 0)
        {
            c[k] = c[k] * (T(1) - tau);
        }
        else if (tau != T(0))
        {
            T tmp = T(0);
#pragma unroll
            for (int i = 0; i < len; ++i)
            {
                const T p = qr[(k + 1 + i) * N + k] * c[k + 1 + i];
                tmp = (i == 0) ? p : tmp + p;
            }
            tmp = tmp + c[k];
            c[k] = c[k] - tau * tmp;
#pragma unroll
            for (int i = 0; i < len; ++i)
                c[k + 1 + i] = c[k + 1 + i] - (tau * qr[(k + 1 + i) * N + k]) * tmp;
        }
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i)
    {
        if (i < nz && c[i] != T(0))
        {
            c[i] = c[i] / qr[i * N + i];
#pragma unroll
            for (int s = 0; s < i; ++s)
                c[s] = c[s] - c[i] * qr[s * N + i];
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
    {
        const T val = (i < nz) ? c[i] : T(0);
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (perm[i] == j)
                x[j] = val;
    }
}


template <int N>
__device__ __forceinline__ void cpqr_solve(const float *A, const float *b, float *x)
{
    cpqr_solve_t<float, N>(A, b, x);
}

template <typename T>
__device__ __forceinline__ T qef_err4_t(const T Q[16], const T p[4])
{
    T r[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const T col[4] = {Q[0 * 4 + j], Q[1 * 4 + j], Q[2 * 4 + j], Q[3 * 4 + j]};
        r[j] = Arith<T>::dot4(p, col);
    }
    return Arith<T>::dot4(r, p);
}

// Regularisation toward the mass point (flexible_dual_grid.cpp:780-792): Q += (rw*cnt) * Qreg.
template <typename T>
__device__ __forceinline__ void regularize_t(const T q_in[10], const T mean[3], T cnt, T rw, T q[10])
{
#pragma unroll
    for (int i = 0; i < 10; ++i)
        q[i] = q_in[i];
    if (rw > T(0))
    {
        const T p0 = mean[0] / cnt, p1 = mean[1] / cnt, p2 = mean[2] / cnt;
        const T s = rw * cnt;
        const T pp = Arith<T>::dot3(p0, p1, p2, p0, p1, p2);
        q[0] = q[0] + s * T(1);
        q[1] = q[1] + s * T(0);
        q[2] = q[2] + s * T(0);
        q[3] = q[3] + s * (-p0);
        q[4] = q[4] + s * T(1);
        q[5] = q[5] + s * T(0);
        q[6] = q[6] + s * (-p1);
        q[7] = q[7] + s * T(1);
        q[8] = q[8] + s * (-p2);
        q[9] = q[9] + s * pp;
    }
}

__device__ __forceinline__ void regularize(const float q_in[10], const float mean[3], float cnt, float rw, float q[10])
{
    regularize_t<float>(q_in, mean, cnt, rw, q);
}

template <typename T>
__device__ __forceinline__ void voxel_box_t(const int coord[3], const Grid &g, T mn[3], T mx[3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i)
    {
        mn[i] = (T)((float)coord[i] * g.vs[i]);
        mx[i] = (T)((float)(coord[i] + 1) * g.vs[i]);
    }
}

// Unconstrained minimiser A v = -b (flexible_dual_grid.cpp:795-797); true if it lies in the voxel box.
template <typename T>
__device__ __forceinline__ bool solve_unconstrained_t(const int coord[3], const Grid &g, const T q[10], T v[3], T *rdiag = nullptr)
{
    const T A[9] = {q[0], q[1], q[2], q[1], q[4], q[5], q[2], q[5], q[7]};
    const T bb[3] = {-q[3], -q[6], -q[8]};
    cpqr_solve_t<T, 3>(A, bb, v, rdiag);
    T mn[3], mx[3];
    voxel_box_t<T>(coord, g, mn, mx);
    return v[0] >= mn[0] && v[0] <= mx[0] && v[1] >= mn[1] && v[1] <= mx[1] && v[2] >= mn[2] && v[2] <= mx[2];
}

__device__ __forceinline__ bool solve_unconstrained(const int coord[3], const Grid &g, const float q[10], float v[3])
{
    return solve_unconstrained_t<float>(coord, g, q, v);
}

// Constrained search over the box faces, edges and corners (flexible_dual_grid.cpp:799-979),
// starting from the unconstrained solution, strict `<` in the reference order.
template <typename T>
__device__ __forceinline__ void solve_constrained_t(const int coord[3], const Grid &g, const T q[10], T v[3])
{
    solve_unconstrained_t<T>(coord, g, q, v);
    T mn[3], mx[3];
    voxel_box_t<T>(coord, g, mn, mx);
    const T Q[16] = {q[0], q[1], q[2], q[3], q[1], q[4], q[5], q[6], q[2], q[5], q[7], q[8], q[3], q[6], q[8], q[9]};
    T best = (T)__int_as_float(0x7f800000);
#pragma unroll 1
    for (int fa = 0; fa < 3; ++fa)
    {
        const int a1 = (fa + 1) % 3, a2 = (fa + 2) % 3;
        const T A2[4] = {Q[a1 * 4 + a1], Q[a1 * 4 + a2], Q[a2 * 4 + a1], Q[a2 * 4 + a2]};
        const T B2[4] = {Q[a1 * 4 + fa], Q[a1 * 4 + 3], Q[a2 * 4 + fa], Q[a2 * 4 + 3]};
#pragma unroll 1
        for (int bound = 0; bound < 2; ++bound)
        {
            const T fv = bound == 0 ? mn[fa] : mx[fa];
            const T rhs[2] = {(-B2[0]) * fv + (-B2[1]) * T(1), (-B2[2]) * fv + (-B2[3]) * T(1)};
            T x2[2];
            cpqr_solve_t<T, 2>(A2, rhs, x2);
            if (x2[0] >= mn[a1] && x2[0] <= mx[a1] && x2[1] >= mn[a2] && x2[1] <= mx[a2])
            {
                T p[4];
                p[fa] = fv;
                p[a1] = x2[0];
                p[a2] = x2[1];
                p[3] = T(1);
                const T err = qef_err4_t<T>(Q, p);
                if (err < best)
                {
                    best = err;
                    v[0] = p[0];
                    v[1] = p[1];
                    v[2] = p[2];
                }
            }
        }
    }
#pragma unroll 1
    for (int fr = 0; fr < 3; ++fr)
    {
        const int a1 = (fr + 1) % 3, a2 = (fr + 2) % 3;
        const T a = Q[fr * 4 + fr];
        const T b0 = Q[fr * 4 + a1], b1 = Q[fr * 4 + a2], b2 = Q[fr * 4 + 3];
#pragma unroll 1
        for (int cc = 0; cc < 4; ++cc)
        {
            const T u1 = (cc >> 1) == 0 ? mn[a1] : mx[a1];
            const T u2 = (cc & 1) == 0 ? mn[a2] : mx[a2];
            const T xf = -(Arith<T>::dot3(b0, b1, b2, u1, u2, T(1))) / a;
            if (xf >= mn[fr] && xf <= mx[fr])
            {
                T p[4];
                p[fr] = xf;
                p[a1] = u1;
                p[a2] = u2;
                p[3] = T(1);
                const T err = qef_err4_t<T>(Q, p);
                if (err < best)
                {
                    best = err;
                    v[0] = p[0];
                    v[1] = p[1];
                    v[2] = p[2];
                }
            }
        }
    }
#pragma unroll 1
    for (int cn = 0; cn < 8; ++cn)
    {
        T p[4];
        p[0] = (cn & 4) ? mn[0] : mx[0];
        p[1] = (cn & 2) ? mn[1] : mx[1];
        p[2] = (cn & 1) ? mn[2] : mx[2];
        p[3] = T(1);
        const T err = qef_err4_t<T>(Q, p);
        if (err < best)
        {
            best = err;
            v[0] = p[0];
            v[1] = p[1];
            v[2] = p[2];
        }
    }
}

__device__ __forceinline__ void solve_constrained(const int coord[3], const Grid &g, const float q[10], float v[3])
{
    solve_constrained_t<float>(coord, g, q, v);
}

} // namespace ovx
