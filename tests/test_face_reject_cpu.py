"""The whole-box rejection of the face stage (face_box_rejects in
fdg_device.cuh) is exact: whenever it rejects a box, the per-voxel test
(face_test_c) fails for every voxel of the box.

Both are restated here in numpy float32, one rounding per operation as the
device code computes them (the library is built without FMA contraction).
The property rests only on IEEE rounding being monotone, so it must hold for
any coefficients: the cases below draw them at random, with offsets placed
around the box's value range so that both outcomes occur often.
"""
import numpy as np

F = np.float32


def _dot3(a0, a1, a2, b0, b1, b2):
    return F(a0) * F(b0) + (F(a1) * F(b1) + F(a2) * F(b2))


def _dot2(a0, a1, b0, b1):
    return F(a0) * F(b0) + F(a1) * F(b1)


def voxel_pass(C, vs, x, y, z):
    """face_test_c at voxels (x, y, z) (arrays): True where the test passes."""
    p0, p1, p2 = F(vs[0]) * x.astype(F), F(vs[1]) * y.astype(F), F(vs[2]) * z.astype(F)
    nd = _dot3(C[0], C[1], C[2], p0, p1, p2)
    ok = ~((nd + C[3]) * (nd + C[4]) > F(0))
    for k in range(3):
        ok &= ~(_dot2(C[5 + 2 * k], C[6 + 2 * k], p0, p1) + C[11 + k] < F(0))
        ok &= ~(_dot2(C[14 + 2 * k], C[15 + 2 * k], p1, p2) + C[20 + k] < F(0))
        ok &= ~(_dot2(C[23 + 2 * k], C[24 + 2 * k], p2, p0) + C[29 + k] < F(0))
    return ok


def box_rejects(C, vs, lo, hi):
    def pick(c, a, want_max):
        i = hi[a] - 1 if (c >= F(0)) == want_max else lo[a]
        return F(vs[a]) * F(i)

    nlo = _dot3(C[0], C[1], C[2], pick(C[0], 0, False), pick(C[1], 1, False), pick(C[2], 2, False))
    ul, wl = nlo + C[3], nlo + C[4]
    if ul > 0 and wl > 0 and ul * wl > 0:
        return True
    nhi = _dot3(C[0], C[1], C[2], pick(C[0], 0, True), pick(C[1], 1, True), pick(C[2], 2, True))
    uh, wh = nhi + C[3], nhi + C[4]
    if uh < 0 and wh < 0 and uh * wh > 0:
        return True
    for k in range(3):
        if _dot2(C[5 + 2 * k], C[6 + 2 * k], pick(C[5 + 2 * k], 0, True), pick(C[6 + 2 * k], 1, True)) + C[11 + k] < 0:
            return True
        if _dot2(C[14 + 2 * k], C[15 + 2 * k], pick(C[14 + 2 * k], 1, True), pick(C[15 + 2 * k], 2, True)) + C[20 + k] < 0:
            return True
        if _dot2(C[23 + 2 * k], C[24 + 2 * k], pick(C[23 + 2 * k], 2, True), pick(C[24 + 2 * k], 0, True)) + C[29 + k] < 0:
            return True
    return False


def _case(rng):
    vs = rng.uniform(1e-3, 1.0, 3).astype(F)
    lo = rng.integers(-600, 600, 3)
    hi = lo + rng.integers(1, 9, 3)
    C = rng.standard_normal(32).astype(F)
    C[rng.random(32) < 0.1] = F(0)           # zero coefficients, both signs
    C[rng.random(32) < 0.05] *= F(-0.0)
    # offsets near minus the coefficient terms at a random voxel of the box, so that
    # the tests sit close to their thresholds there
    c = lo + rng.integers(0, hi - lo)
    p = vs * c.astype(F)
    nd = _dot3(C[0], C[1], C[2], p[0], p[1], p[2])
    # half the cases pass at that voxel by a small margin (slab straddled,
    # half-planes on the inner side), the others sit at random near the thresholds
    inside = rng.random() < 0.5
    eps = 1e-6
    if inside:
        C[3] = -nd + F(abs(nd) * eps + 1e-12)
        C[4] = -nd - F(abs(nd) * eps + 1e-12)
    else:
        C[3] = -nd + F(rng.standard_normal() * abs(nd) * eps)
        C[4] = -nd + F(rng.standard_normal() * abs(nd) * eps)

    def offset(val):
        if inside:
            return -val + F(abs(val) * eps + 1e-12)
        return -val * F(1 + rng.standard_normal() * eps)

    for k in range(3):
        C[11 + k] = offset(_dot2(C[5 + 2 * k], C[6 + 2 * k], p[0], p[1]))
        C[20 + k] = offset(_dot2(C[14 + 2 * k], C[15 + 2 * k], p[1], p[2]))
        C[29 + k] = offset(_dot2(C[23 + 2 * k], C[24 + 2 * k], p[2], p[0]))
    return C, vs, lo, hi


def test_rejection_is_exact():
    rng = np.random.default_rng(7)
    rejected = kept_with_hits = 0
    for _ in range(3000):
        C, vs, lo, hi = _case(rng)
        x, y, z = np.meshgrid(*[np.arange(lo[a], hi[a]) for a in range(3)], indexing="ij")
        ok = voxel_pass(C, vs, x, y, z)
        if box_rejects(C, vs, lo, hi):
            rejected += 1
            assert not ok.any(), "a rejected box holds a voxel that passes the per-voxel test"
        elif ok.any():
            kept_with_hits += 1
    # both outcomes occur, so the property was exercised
    assert rejected > 300 and kept_with_hits > 10, (rejected, kept_with_hits)


def test_box_with_a_passing_voxel_is_kept():
    """The converse direction of the same property: a box holding a voxel that
    passes the per-voxel test is never rejected."""
    rng = np.random.default_rng(3)
    for _ in range(200):
        C, vs, lo, hi = _case(rng)
        x, y, z = np.meshgrid(*[np.arange(lo[a], hi[a]) for a in range(3)], indexing="ij")
        if voxel_pass(C, vs, x, y, z).any():
            assert not box_rejects(C, vs, lo, hi)
