/*
 * fdg_oracle_impl.h -- body of the CPU oracle, instantiated twice by
 * fdg_oracle.c: once with REAL=float (the exact restatement of the reference
 * CPU path) and once with REAL=double (same geometry decisions, FP64
 * accumulation and solve; used only for error statistics).
 *
 * TEST INFRASTRUCTURE: this file is the checker for the CUDA path.  Nothing in
 * the product links it.
 *
 * Reference semantics followed (paths relative to the reference project):
 *   src/convert/flexible_dual_grid.cpp:158-285  intersect_qef
 *   src/convert/flexible_dual_grid.cpp:287-415  face_qef
 *   src/convert/flexible_dual_grid.cpp:417-524  boundry_qef
 *   src/convert/flexible_dual_grid.cpp:660-992  mesh_to_flexible_dual_grid_cpu
 *   src/convert/flexible_dual_grid.cpp:80-156   intersect_occ
 */

#ifndef REAL
#error "define REAL and FN() before including fdg_oracle_impl.h"
#endif

/* ------------------------------------------------------------------ */
/* Quadric helpers.  Q is a symmetric 4x4 stored as 10 upper entries:   */
/* q00 q01 q02 q03 q11 q12 q13 q22 q23 q33.                             */
/* ------------------------------------------------------------------ */

static inline REAL FN(dot3)(REAL a0, REAL a1, REAL a2, REAL b0, REAL b1, REAL b2)
{
    /* Eigen fixed-size 3-vector reduction (non-vectorised unroller): a0*b0 + (a1*b1 + a2*b2). */
    return a0 * b0 + (a1 * b1 + a2 * b2);
}

static inline REAL FN(dot4v)(const REAL a[4], const REAL b[4])
{
    /* Eigen 4-wide packet reduction (predux of one SSE packet): (e0+e2)+(e1+e3). */
    return (a[0] * b[0] + a[2] * b[2]) + (a[1] * b[1] + a[3] * b[3]);
}

static inline void FN(q_to_dense)(const REAL q[10], REAL Q[16])
{
    Q[0] = q[0]; Q[1] = q[1]; Q[2] = q[2]; Q[3] = q[3];
    Q[4] = q[1]; Q[5] = q[4]; Q[6] = q[5]; Q[7] = q[6];
    Q[8] = q[2]; Q[9] = q[5]; Q[10] = q[7]; Q[11] = q[8];
    Q[12] = q[3]; Q[13] = q[6]; Q[14] = q[8]; Q[15] = q[9];
}

/* p^T Q p, evaluated as Eigen evaluates `p.transpose() * Q * p` for Vector4f/Matrix4f
 * (flexible_dual_grid.cpp:836): row r = p^T Q by per-column packet reductions, then r.p. */
static inline REAL FN(qef_err4)(const REAL Q[16], const REAL p[4])
{
    REAL r[4];
    for (int j = 0; j < 4; ++j)
    {
        const REAL col[4] = {Q[0 * 4 + j], Q[1 * 4 + j], Q[2 * 4 + j], Q[3 * 4 + j]};
        r[j] = FN(dot4v)(p, col);
    }
    return FN(dot4v)(r, p);
}

/* ------------------------------------------------------------------ */
/* Column-pivoting Householder QR solve (Eigen ColPivHouseholderQR     */
/* algorithm: LAPACK xGEQPF-style pivoting with stable norm downdates,  */
/* rank = number of pivots above the threshold_helper test).            */
/* A is row-major n x n, n in {2,3}.                                    */
/* ------------------------------------------------------------------ */
static void FN(cpqr_solve)(int n, const REAL *A, const REAL *b, REAL *x)
{
    REAL qr[9], c[3], hcoeff[3], nu[3], nd[3];
    int perm[3];
    const REAL eps = REAL_EPS;
    for (int i = 0; i < n * n; ++i)
        qr[i] = A[i];
    for (int i = 0; i < n; ++i)
    {
        c[i] = b[i];
        perm[i] = i;
        x[i] = 0;
    }
    for (int j = 0; j < n; ++j)
    {
        /* fixed-size column norm: n=3 -> a0^2 + (a1^2 + a2^2), n=2 -> a0^2 + a1^2 */
        REAL s;
        if (n == 3)
            s = qr[0 * 3 + j] * qr[0 * 3 + j] + (qr[1 * 3 + j] * qr[1 * 3 + j] + qr[2 * 3 + j] * qr[2 * 3 + j]);
        else
            s = qr[0 * 2 + j] * qr[0 * 2 + j] + qr[1 * 2 + j] * qr[1 * 2 + j];
        nd[j] = nu[j] = REAL_SQRT(s);
    }
    REAL maxn = nu[0];
    for (int j = 1; j < n; ++j)
        if (nu[j] > maxn)
            maxn = nu[j];
    const REAL th = (maxn * eps) * (maxn * eps) / (REAL)n;
    const REAL downdate_th = REAL_SQRT(eps);
    int nz = n;

    for (int k = 0; k < n; ++k)
    {
        int bi = k;
        REAL bv = nu[k];
        for (int j = k + 1; j < n; ++j)
            if (nu[j] > bv)
            {
                bv = nu[j];
                bi = j;
            }
        if (nz == n && bv * bv < th * (REAL)(n - k))
            nz = k;
        if (bi != k)
        {
            for (int r = 0; r < n; ++r)
            {
                REAL t = qr[r * n + k];
                qr[r * n + k] = qr[r * n + bi];
                qr[r * n + bi] = t;
            }
            REAL t = nu[k]; nu[k] = nu[bi]; nu[bi] = t;
            t = nd[k]; nd[k] = nd[bi]; nd[bi] = t;
            int ti = perm[k]; perm[k] = perm[bi]; perm[bi] = ti;
        }
        /* Householder reflector for column k, rows k..n-1. */
        const int len = n - k - 1;
        const REAL c0 = qr[k * n + k];
        REAL tsq = 0;
        for (int i = 0; i < len; ++i)
        {
            const REAL e = qr[(k + 1 + i) * n + k];
            tsq = (i == 0) ? e * e : tsq + e * e;
        }
        REAL tau, beta;
        if (tsq <= REAL_MIN)
        {
            tau = 0;
            beta = c0;
            for (int i = 0; i < len; ++i)
                qr[(k + 1 + i) * n + k] = 0;
        }
        else
        {
            beta = REAL_SQRT(c0 * c0 + tsq);
            if (c0 >= 0)
                beta = -beta;
            const REAL den = c0 - beta;
            for (int i = 0; i < len; ++i)
                qr[(k + 1 + i) * n + k] = qr[(k + 1 + i) * n + k] / den;
            tau = (beta - c0) / beta;
        }
        qr[k * n + k] = beta;
        hcoeff[k] = tau;
        /* apply to the trailing columns k+1..n-1 (rows k..n-1) */
        if (len > 0 && tau != 0)
        {
            for (int j = k + 1; j < n; ++j)
            {
                REAL tmp = 0;
                for (int i = 0; i < len; ++i)
                {
                    const REAL prod = qr[(k + 1 + i) * n + k] * qr[(k + 1 + i) * n + j];
                    tmp = (i == 0) ? prod : tmp + prod;
                }
                tmp = tmp + qr[k * n + j];
                qr[k * n + j] = qr[k * n + j] - tau * tmp;
                for (int i = 0; i < len; ++i)
                    qr[(k + 1 + i) * n + j] = qr[(k + 1 + i) * n + j] - (tau * qr[(k + 1 + i) * n + k]) * tmp;
            }
        }
        /* norm downdates */
        for (int j = k + 1; j < n; ++j)
        {
            if (nu[j] != 0)
            {
                REAL temp = REAL_ABS(qr[k * n + j]) / nu[j];
                temp = (1 + temp) * (1 - temp);
                temp = temp < 0 ? 0 : temp;
                const REAL ratio = nu[j] / nd[j];
                const REAL temp2 = temp * (ratio * ratio);
                if (temp2 <= downdate_th)
                {
                    REAL s = 0;
                    for (int r = k + 1; r < n; ++r)
                    {
                        const REAL e = qr[r * n + j];
                        s = (r == k + 1) ? e * e : s + e * e;
                    }
                    nd[j] = nu[j] = REAL_SQRT(s);
                }
                else
                {
                    nu[j] = nu[j] * REAL_SQRT(temp);
                }
            }
        }
    }

    if (nz == 0)
        return; /* x already zero */

    /* c <- Q^T c using the first nz reflectors, in order */
    for (int k = 0; k < nz; ++k)
    {
        const int len = n - k - 1;
        const REAL tau = hcoeff[k];
        if (len == 0)
        {
            c[k] = c[k] * (1 - tau);
        }
        else if (tau != 0)
        {
            REAL tmp = 0;
            for (int i = 0; i < len; ++i)
            {
                const REAL prod = qr[(k + 1 + i) * n + k] * c[k + 1 + i];
                tmp = (i == 0) ? prod : tmp + prod;
            }
            tmp = tmp + c[k];
            c[k] = c[k] - tau * tmp;
            for (int i = 0; i < len; ++i)
                c[k + 1 + i] = c[k + 1 + i] - (tau * qr[(k + 1 + i) * n + k]) * tmp;
        }
    }
    /* column-oriented upper-triangular back substitution on the leading nz x nz block */
    for (int i = nz - 1; i >= 0; --i)
    {
        if (c[i] != 0)
        {
            c[i] = c[i] / qr[i * n + i];
            for (int s = 0; s < i; ++s)
                c[s] = c[s] - c[i] * qr[s * n + i];
        }
    }
    for (int i = 0; i < nz; ++i)
        x[perm[i]] = c[i];
    for (int i = nz; i < n; ++i)
        x[perm[i]] = 0;
}

/* ------------------------------------------------------------------ */
/* Dual vertex solve for one voxel (flexible_dual_grid.cpp:766-983).     */
/* q: accumulated quadric (10 entries), mean: summed intersection points */
/* ------------------------------------------------------------------ */
static void FN(solve_voxel)(const int32_t coord[3], const float vs[3], const REAL q_in[10],
                            const REAL mean[3], REAL cnt, float rw, REAL out[3])
{
    REAL q[10];
    for (int i = 0; i < 10; ++i)
        q[i] = q_in[i];
    float mn[3], mx[3];
    for (int i = 0; i < 3; ++i)
    {
        mn[i] = (float)coord[i] * vs[i];
        mx[i] = (float)(coord[i] + 1) * vs[i];
    }
    if (rw > 0.0f)
    {
        const REAL p0 = mean[0] / cnt, p1 = mean[1] / cnt, p2 = mean[2] / cnt;
        const REAL s = (REAL)rw * cnt;
        const REAL pp = FN(dot3)(p0, p1, p2, p0, p1, p2);
        const REAL zero = 0, one = 1;
        q[0] = q[0] + s * one;
        q[1] = q[1] + s * zero;
        q[2] = q[2] + s * zero;
        q[3] = q[3] + s * (-p0);
        q[4] = q[4] + s * one;
        q[5] = q[5] + s * zero;
        q[6] = q[6] + s * (-p1);
        q[7] = q[7] + s * one;
        q[8] = q[8] + s * (-p2);
        q[9] = q[9] + s * pp;
    }
    REAL Q[16];
    FN(q_to_dense)(q, Q);
    const REAL A[9] = {Q[0], Q[1], Q[2], Q[4], Q[5], Q[6], Q[8], Q[9], Q[10]};
    const REAL bb[3] = {-Q[3], -Q[7], -Q[11]};
    REAL v[3];
    FN(cpqr_solve)(3, A, bb, v);

    if (!(v[0] >= mn[0] && v[0] <= mx[0] && v[1] >= mn[1] && v[1] <= mx[1] && v[2] >= mn[2] && v[2] <= mx[2]))
    {
        REAL best = (REAL)INFINITY;
        /* single constraint: fix one axis at min or max, solve the 2x2 face system */
        for (int fa = 0; fa < 3; ++fa)
        {
            const int a1 = (fa + 1) % 3, a2 = (fa + 2) % 3;
            const REAL A2[4] = {Q[a1 * 4 + a1], Q[a1 * 4 + a2], Q[a2 * 4 + a1], Q[a2 * 4 + a2]};
            const REAL B2[4] = {Q[a1 * 4 + fa], Q[a1 * 4 + 3], Q[a2 * 4 + fa], Q[a2 * 4 + 3]};
            for (int bound = 0; bound < 2; ++bound)
            {
                const REAL fv = bound == 0 ? (REAL)mn[fa] : (REAL)mx[fa];
                const REAL one = 1;
                const REAL rhs[2] = {(-B2[0]) * fv + (-B2[1]) * one, (-B2[2]) * fv + (-B2[3]) * one};
                REAL x2[2];
                FN(cpqr_solve)(2, A2, rhs, x2);
                if (x2[0] >= mn[a1] && x2[0] <= mx[a1] && x2[1] >= mn[a2] && x2[1] <= mx[a2])
                {
                    REAL p[4];
                    p[fa] = fv;
                    p[a1] = x2[0];
                    p[a2] = x2[1];
                    p[3] = 1;
                    const REAL err = FN(qef_err4)(Q, p);
                    if (err < best)
                    {
                        best = err;
                        v[0] = p[0]; v[1] = p[1]; v[2] = p[2];
                    }
                }
            }
        }
        /* two constraints: fix two axes at box bounds, 1D minimiser along the free axis */
        for (int fr = 0; fr < 3; ++fr)
        {
            const int a1 = (fr + 1) % 3, a2 = (fr + 2) % 3;
            const REAL a = Q[fr * 4 + fr];
            const REAL b0 = Q[fr * 4 + a1], b1 = Q[fr * 4 + a2], b2 = Q[fr * 4 + 3];
            for (int c1 = 0; c1 < 2; ++c1)
                for (int c2 = 0; c2 < 2; ++c2)
                {
                    const REAL u1 = c1 == 0 ? (REAL)mn[a1] : (REAL)mx[a1];
                    const REAL u2 = c2 == 0 ? (REAL)mn[a2] : (REAL)mx[a2];
                    const REAL xf = -(FN(dot3)(b0, b1, b2, u1, u2, (REAL)1)) / a;
                    if (xf >= mn[fr] && xf <= mx[fr])
                    {
                        REAL p[4];
                        p[fr] = xf;
                        p[a1] = u1;
                        p[a2] = u2;
                        p[3] = 1;
                        const REAL err = FN(qef_err4)(Q, p);
                        if (err < best)
                        {
                            best = err;
                            v[0] = p[0]; v[1] = p[1]; v[2] = p[2];
                        }
                    }
                }
        }
        /* three constraints: the 8 box corners (index 0 selects the max corner) */
        for (int cx = 0; cx < 2; ++cx)
            for (int cy = 0; cy < 2; ++cy)
                for (int cz = 0; cz < 2; ++cz)
                {
                    REAL p[4];
                    p[0] = cx ? (REAL)mn[0] : (REAL)mx[0];
                    p[1] = cy ? (REAL)mn[1] : (REAL)mx[1];
                    p[2] = cz ? (REAL)mn[2] : (REAL)mx[2];
                    p[3] = 1;
                    const REAL err = FN(qef_err4)(Q, p);
                    if (err < best)
                    {
                        best = err;
                        v[0] = p[0]; v[1] = p[1]; v[2] = p[2];
                    }
                }
    }
    out[0] = v[0];
    out[1] = v[1];
    out[2] = v[2];
}

/* ------------------------------------------------------------------ */
/* Accumulator state shared by the three quadric stages.                 */
/* ------------------------------------------------------------------ */
typedef struct FN(acc)
{
    vox_map map;
    int64_t n, cap;
    int32_t *vox;
    REAL *mean;
    REAL *cnt;
    uint8_t *flag;
    REAL *qef;
    REAL tri_q[10]; /* quadric of the triangle being scanned */
    int oom;
} FN(acc);

static void FN(acc_grow)(FN(acc) *a)
{
    if (a->n < a->cap)
        return;
    int64_t nc = a->cap ? a->cap * 2 : 1024;
    a->vox = (int32_t *)realloc(a->vox, (size_t)nc * 3 * sizeof(int32_t));
    a->mean = (REAL *)realloc(a->mean, (size_t)nc * 3 * sizeof(REAL));
    a->cnt = (REAL *)realloc(a->cnt, (size_t)nc * sizeof(REAL));
    a->flag = (uint8_t *)realloc(a->flag, (size_t)nc * 3);
    a->qef = (REAL *)realloc(a->qef, (size_t)nc * 10 * sizeof(REAL));
    if (!a->vox || !a->mean || !a->cnt || !a->flag || !a->qef)
        a->oom = 1;
    a->cap = nc;
}

/* Event callback for the intersection stage (flexible_dual_grid.cpp:243-271). */
static void FN(on_event)(void *ctx, const int32_t coord[3], int ax2, int dx, int dy, const double pt[3])
{
    FN(acc) *a = (FN(acc) *)ctx;
    if (a->oom)
        return;
    const uint64_t key = map_key(coord);
    int64_t idx = map_find(&a->map, key);
#if REAL_IS_FLOAT
    const REAL p0 = (float)pt[0], p1 = (float)pt[1], p2 = (float)pt[2];
#else
    const REAL p0 = pt[0], p1 = pt[1], p2 = pt[2];
#endif
    if (idx < 0)
    {
        FN(acc_grow)(a);
        if (a->oom)
            return;
        idx = a->n++;
        if (map_insert(&a->map, key, idx) != 0)
        {
            a->oom = 1;
            return;
        }
        a->vox[idx * 3 + 0] = coord[0];
        a->vox[idx * 3 + 1] = coord[1];
        a->vox[idx * 3 + 2] = coord[2];
        a->mean[idx * 3 + 0] = p0;
        a->mean[idx * 3 + 1] = p1;
        a->mean[idx * 3 + 2] = p2;
        a->cnt[idx] = 1;
        a->flag[idx * 3 + 0] = a->flag[idx * 3 + 1] = a->flag[idx * 3 + 2] = 0;
        for (int i = 0; i < 10; ++i)
            a->qef[idx * 10 + i] = a->tri_q[i];
    }
    else
    {
        a->mean[idx * 3 + 0] = a->mean[idx * 3 + 0] + p0;
        a->mean[idx * 3 + 1] = a->mean[idx * 3 + 1] + p1;
        a->mean[idx * 3 + 2] = a->mean[idx * 3 + 2] + p2;
        a->cnt[idx] = a->cnt[idx] + 1;
        for (int i = 0; i < 10; ++i)
            a->qef[idx * 10 + i] = a->qef[idx * 10 + i] + a->tri_q[i];
    }
    if (dx == 0 && dy == 0)
        a->flag[idx * 3 + ax2] = 1;
}

/* Plane quadric of a triangle (flexible_dual_grid.cpp:180-185 / :305-311):
 * n = normalize(cross(v1-v0, v2-v1)) in float, plane = (n, -n.v0), Q = plane plane^T. */
static void FN(triangle_quadric)(const float v[3][3], REAL q[10])
{
#if REAL_IS_FLOAT
    float n[3];
    tri_normal(v, n);
    const float d = -dot3f(n[0], n[1], n[2], v[0][0], v[0][1], v[0][2]);
    const REAL p[4] = {n[0], n[1], n[2], d};
#else
    double n[3];
    tri_normal_f64(v, n);
    const double d = -FN(dot3)(n[0], n[1], n[2], v[0][0], v[0][1], v[0][2]);
    const REAL p[4] = {n[0], n[1], n[2], d};
#endif
    q[0] = p[0] * p[0]; q[1] = p[0] * p[1]; q[2] = p[0] * p[2]; q[3] = p[0] * p[3];
    q[4] = p[1] * p[1]; q[5] = p[1] * p[2]; q[6] = p[1] * p[3];
    q[7] = p[2] * p[2]; q[8] = p[2] * p[3];
    q[9] = p[3] * p[3];
}

/* ------------------------------------------------------------------ */
/* Full pipeline (flexible_dual_grid.cpp:660-992).                       */
/* ------------------------------------------------------------------ */
int FN(fdg_oracle_mesh_to_fdg)(const float *verts, int64_t nv, const int32_t *faces, int64_t nf,
                               const float vs[3], const int32_t grid_range[6],
                               float fw, float bw, float rw, fdg_oracle_out *out)
{
    memset(out, 0, sizeof(*out));
    const int32_t gmin[3] = {grid_range[0], grid_range[1], grid_range[2]};
    const int32_t gmax[3] = {grid_range[3], grid_range[4], grid_range[5]};
    for (int64_t i = 0; i < nf * 3; ++i)
        if (faces[i] < 0 || faces[i] >= nv)
            return FDG_ORACLE_BAD_INDEX;
    map_set_grid(gmin, gmax);

    FN(acc) a;
    memset(&a, 0, sizeof(a));
    if (map_init(&a.map, 1 << 12) != 0)
        return FDG_ORACLE_OOM;

    /* Intersection stage: triangle order, axes 0,1,2, scanline events. */
    for (int64_t f = 0; f < nf; ++f)
    {
        float v[3][3];
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c)
                v[k][c] = verts[(int64_t)faces[f * 3 + k] * 3 + c];
        FN(triangle_quadric)(v, a.tri_q);
        scan_triangle(v, vs, gmin, gmax, FN(on_event), &a);
        if (a.oom)
            break;
    }

    /* Face stage (only a gate on face_weight; the quadric is added unscaled). */
    if (!a.oom && fw > 0.0f)
    {
        for (int64_t f = 0; f < nf; ++f)
        {
            float v[3][3];
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c)
                    v[k][c] = verts[(int64_t)faces[f * 3 + k] * 3 + c];
            REAL q[10];
            FN(triangle_quadric)(v, q);
            face_setup fs;
            face_prepare(v, vs, gmin, gmax, &fs);
            for (int z = fs.bmin[2]; z < fs.bmax[2]; ++z)
                for (int y = fs.bmin[1]; y < fs.bmax[1]; ++y)
                    for (int x = fs.bmin[0]; x < fs.bmax[0]; ++x)
                    {
                        if (!face_test(&fs, vs, x, y, z))
                            continue;
                        const int32_t c[3] = {x, y, z};
                        const int64_t idx = map_find(&a.map, map_key(c));
                        if (idx >= 0)
                            for (int i = 0; i < 10; ++i)
                                a.qef[idx * 10 + i] = a.qef[idx * 10 + i] + q[i];
                    }
        }
    }

    /* Boundary stage: undirected edges used by exactly one face, in sorted (min,max) order. */
    if (!a.oom && bw > 0.0f)
    {
        int64_t ne = 0;
        uint64_t *bedges = boundary_edges(faces, nf, &ne);
        if (!bedges && nf > 0)
            a.oom = 1;
        out->num_boundary_edges = ne;
        for (int64_t e = 0; e < ne && !a.oom; ++e)
        {
            const int32_t i0 = (int32_t)(bedges[e] >> 32), i1 = (int32_t)(bedges[e] & 0xffffffffu);
            const float p0[3] = {verts[(int64_t)i0 * 3 + 0], verts[(int64_t)i0 * 3 + 1], verts[(int64_t)i0 * 3 + 2]};
            const float p1[3] = {verts[(int64_t)i1 * 3 + 0], verts[(int64_t)i1 * 3 + 1], verts[(int64_t)i1 * 3 + 2]};
            float bq[10];
            double bq64[10];
            int32_t walk[3];
            dda_state st;
            if (!boundary_prepare(p0, p1, vs, bq, bq64, &st))
                continue;
            REAL wq[10];
            for (int i = 0; i < 10; ++i)
#if REAL_IS_FLOAT
                wq[i] = bw * bq[i];
#else
                wq[i] = (double)bw * bq64[i];
#endif
            while (dda_next(&st, walk))
            {
                if (walk[0] < gmin[0] || walk[0] >= gmax[0] || walk[1] < gmin[1] || walk[1] >= gmax[1] ||
                    walk[2] < gmin[2] || walk[2] >= gmax[2])
                    continue;
                const int64_t idx = map_find(&a.map, map_key(walk));
                if (idx >= 0)
                    for (int i = 0; i < 10; ++i)
                        a.qef[idx * 10 + i] = a.qef[idx * 10 + i] + wq[i];
            }
        }
        free(bedges);
    }

    if (a.oom)
    {
        free(a.vox); free(a.mean); free(a.cnt); free(a.flag); free(a.qef);
        map_free(&a.map);
        return FDG_ORACLE_OOM;
    }

    REAL *dual = (REAL *)malloc((size_t)(a.n ? a.n : 1) * 3 * sizeof(REAL));
    for (int64_t i = 0; i < a.n; ++i)
        FN(solve_voxel)(a.vox + i * 3, vs, a.qef + i * 10, a.mean + i * 3, a.cnt[i], rw, dual + i * 3);

    map_free(&a.map);
    out->num_voxels = a.n;
    out->voxels = a.vox;
    out->dual = dual;
    out->intersected = a.flag;
    out->qef = a.qef;
    out->mean_sum = a.mean;
    out->cnt = a.cnt;
    out->elem_size = (int32_t)sizeof(REAL);
    return 0;
}
