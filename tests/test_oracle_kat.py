"""Known-answer tests that pin the CPU oracle.

The reference ships no tests or golden vectors and cannot run here, so the
oracle is pinned by answers derived by hand from the reference source and by a
second, literal pure-Python restatement of the BVH builder on small inputs.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from pulse_b200.layout import node_fields

M32 = 0xFFFFFFFF


def pcg(state):
    """src/utilities.wgsl:67-72 restated with Python integers."""
    state = (state * 747796405 + 2891336453) & M32
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M32
    return state, (word >> 22) ^ word


def test_rand_u_known_answers():
    # state 0: 0*747796405 + 2891336453 = 0xAC564B05; 0xAC564B05 >> 28 = 10, shift 14:
    # (0xAC564B05 >> 14) ^ 0xAC564B05 = 0xAC5667D0... worked with Python integers below.
    st = 0
    st1, w = pcg(st)
    assert st1 == 2891336453
    shifted = 2891336453 >> ((2891336453 >> 28) + 4)
    assert (2891336453 >> 28) == 10 and shifted == 176473
    word = ((shifted ^ 2891336453) * 277803737) & M32
    assert w == (word >> 22) ^ word
    s = np.zeros(1, np.uint32)
    got = [oracle.lib().oracle_rand_u(s.ctypes.data) for _ in range(5)]
    ref, st = [], 0
    for _ in range(5):
        st, r = pcg(st)
        ref.append(r)
    assert got == ref
    assert int(s[0]) == st


def test_rand_f_scale_and_overshoot():
    # rand_f = f32(u32) * bitcast(0x2f800004) = 2^-32 * (1 + 2^-21); f32(2^32-1)
    # rounds to 2^32, so the largest output is 1 + 2^-21 > 1.
    k = np.array([0x2F800004], np.uint32).view(np.float32)[0]
    assert float(k) == 2.0 ** -32 * (1 + 2.0 ** -21)
    top = np.float32(np.float32(4294967295) * k)
    assert top > 1.0 and float(top) == 1 + 2.0 ** -21
    s = np.array([12345], np.uint32)
    st = 12345
    for _ in range(100):
        st, r = pcg(st)
        f = oracle.lib().oracle_rand_f(s.ctypes.data)
        assert np.float32(f) == np.float32(np.float32(r) * k)


def test_sincos_accuracy():
    L = oracle.lib()
    xs = np.concatenate([np.linspace(0, 2 * math.pi * (1 + 2 ** -21), 20001, dtype=np.float32),
                         np.float32([0.0, math.pi / 2, math.pi, 1.5 * math.pi, 1e-8])])
    s = np.zeros(1, np.float32)
    c = np.zeros(1, np.float32)
    err = 0.0
    for x in xs:
        L.oracle_sincos(C.c_float(x), s.ctypes.data, c.ctypes.data)
        err = max(err, abs(float(s[0]) - math.sin(float(x))), abs(float(c[0]) - math.cos(float(x))))
    assert err < 1.2e-7  # about one ulp at 1.0
    L.oracle_sincos(C.c_float(float("nan")), s.ctypes.data, c.ctypes.data)
    assert np.isnan(s[0]) and np.isnan(c[0])


def walk(cdf, offset, count, e):
    """Literal restatement of src/utilities.wgsl:677-691."""
    l, r = offset, offset + count - 1
    while l <= r:
        mid = l + (r - l)
        if cdf[mid] <= e:
            l = mid + 1
        else:
            r = mid - 1
    return min(l, offset + count - 1) - offset


@pytest.mark.parametrize("e,expect", [(0.0, 0), (0.25, 1), (0.3, 1), (0.5, 2), (0.9, 2), (1.0, 2), (1.1, 2),
                                      (-1.0, 0)])
def test_cdf_walk_known_answers(e, expect):
    cdf = np.array([9.0, 0.25, 0.5, 1.0], np.float32)  # offset 1 skips the first entry
    assert walk(cdf, 1, 3, np.float32(e)) == expect
    assert oracle.lib().oracle_cdf_walk(cdf.ctypes.data, 1, 3, C.c_float(e)) == expect


def test_cdf_walk_equals_upper_bound():
    rng = np.random.default_rng(0)
    for _ in range(200):
        n = int(rng.integers(1, 40))
        a = rng.random(n).astype(np.float32)
        a[rng.random(n) < 0.3] = 0.0  # plateaus (zero-area triangles)
        if a.sum() == 0:
            a[0] = 1
        cdf = np.cumsum(a / a.sum(), dtype=np.float32)
        for e in np.concatenate([rng.random(20).astype(np.float32), cdf, [np.float32(1 + 2 ** -21)]]):
            k = oracle.lib().oracle_cdf_walk(cdf.ctypes.data, 0, n, C.c_float(e))
            ub = min(int(np.searchsorted(cdf, e, side="right")), n - 1)
            assert k == ub == walk(cdf, 0, n, e)


def _aabb(o, d, mn, mx, rec_t=1e30):
    f = lambda v: np.asarray(v, np.float32)
    a = [f(o), f(d), f(mn), f(mx)]
    return oracle.lib().oracle_ray_aabb(*(x.ctypes.data for x in a), C.c_float(rec_t))


def test_ray_aabb_known_answers():
    box = ((-1, -1, -1), (1, 1, 1))
    assert _aabb((0, 0, -5), (0, 0, 1), *box) == 4.0
    assert _aabb((0, 0, -5), (0, 0, -1), *box) == np.float32(1e30)      # behind: t_max < 0
    assert _aabb((0, 0, -5), (0, 0, 1), *box, rec_t=3.0) == np.float32(1e30)  # culled by record t
    assert _aabb((0, 0, 0), (0, 0, 1), *box) == -1.0                     # origin inside: t_min < 0
    assert _aabb((0, 3, -5), (0, 0, 1), *box) == np.float32(1e30)       # parallel slab miss (+-inf)


def _tri(o, d, tri):
    f = lambda v: np.asarray(v, np.float32).ravel()
    out = np.zeros(3, np.float32)
    a = [f(o), f(d), f(tri)]
    hit = oracle.lib().oracle_ray_triangle(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, out.ctypes.data)
    return hit, out


def test_ray_triangle_known_answers():
    tri = [(0, 0, 0), (1, 0, 0), (0, 1, 0)]
    hit, tuv = _tri((0.25, 0.25, 1), (0, 0, -1), tri)
    assert hit and tuv.tolist() == [1.0, 0.25, 0.25]
    assert not _tri((0.25, 0.25, 1), (1, 0, 0), tri)[0]         # parallel: |a| < 1e-4
    assert not _tri((0.25, 0.25, 0.0005), (0, 0, -1), tri)[0]   # t = 0.0005 < 0.001
    assert not _tri((0.75, 0.75, 1), (0, 0, -1), tri)[0]        # u + v > 1
    assert not _tri((-0.1, 0.5, 1), (0, 0, -1), tri)[0]         # u < 0
    hit, tuv = _tri((0.5, 0.0, 1), (0, 0, -1), tri)             # on edge v = 0: accepted
    assert hit and tuv[2] == 0.0


def test_inverse4_matches_numpy():
    rng = np.random.default_rng(3)
    for _ in range(50):
        m = np.eye(4)
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        m[:3, :3] = q @ np.diag(rng.uniform(0.5, 2.0, 3))
        m[:3, 3] = rng.uniform(-10, 10, 3)
        cols = m.T.astype(np.float32).ravel()
        inv = oracle.inverse4(cols).reshape(4, 4).T
        np.testing.assert_allclose(inv, np.linalg.inv(m.astype(np.float32).astype(np.float64)), atol=2e-5)


def nine_triangles(x0=0.0):
    """Triangle i has AABB x [x0+i-0.25, x0+i+0.25], y [-0.25, 0.25], z 0 -> centroid (x0+i, 0, 0)."""
    prims = np.zeros((9, 12), np.float32)
    for i in range(9):
        prims[i, 0:3] = (x0 + i - 0.25, -0.25, 0)
        prims[i, 4:7] = (x0 + i + 0.25, -0.25, 0)
        prims[i, 8:11] = (x0 + i, 0.25, 0)
    return prims


def test_blas_nine_triangles_hand_worked():
    """20 bins over centroid x in [0, 8]: tris land in bins 0,2,5,7,10,12,15,17,19.
    Bin and running boxes start as the zero box, so every B box spans x [0, 8.25]
    (area 4.125) and cost(c tris in A) = c*(c-0.5)/2 + (9-c)*4.125, minimal at c=4
    (27.625), first reached at plane 7 -> split x < 0.4f*8 = 3.2.  The two-pointer
    partition leaves [0,1,2,3] and pulls 8,7,6,5 into slot 4 in turn: [0,1,2,3,5,6,7,8,4]."""
    nodes, idx = oracle.build_blas(nine_triangles(), 20, 8)
    assert idx.tolist() == [0, 1, 2, 3, 5, 6, 7, 8, 4]
    mn, a, mx, cnt = node_fields(nodes)
    assert nodes.shape[0] == 3
    assert a.tolist() == [1, 0, 4] and cnt.tolist() == [0, 4, 5]
    assert mn.tolist() == [[-0.25, -0.25, 0], [-0.25, -0.25, 0], [3.75, -0.25, 0]]
    assert mx.tolist() == [[8.25, 0.25, 0], [3.25, 0.25, 0], [8.25, 0.25, 0]]
    # eight triangles stay one leaf (blas.rs:96: tri_count <= 8)
    nodes8, idx8 = oracle.build_blas(nine_triangles()[:8], 20, 8)
    assert nodes8.shape[0] == 1 and idx8.tolist() == list(range(8))


# ----------------------------------------------------------------- builder
def py_build(prims, bins, max_leaf, tlas_bounds=None):
    """Literal pure-Python f32 restatement of build_blas / build_tlas
    (src/scene/blas.rs:44-253, src/scene/tlas.rs:29-263); small inputs only."""
    f = np.float32
    F32MAX = np.finfo(np.float32).max

    def lmin(a, b):
        if a != a:
            return b
        if b != b:
            return a
        if a < b:
            return a
        if b < a:
            return b
        return a if np.signbit(a) else b

    def lmax(a, b):
        if a != a:
            return b
        if b != b:
            return a
        if a > b:
            return a
        if b > a:
            return b
        return b if np.signbit(a) else a

    tlas = tlas_bounds is not None
    n = len(tlas_bounds) if tlas else len(prims)
    if tlas:
        pmin = [tuple(f(v) for v in b[0:3]) for b in tlas_bounds]
        pmax = [tuple(f(v) for v in b[3:6]) for b in tlas_bounds]
        cent = [tuple(f(v) for v in b[6:9]) for b in tlas_bounds]
        grow_pts = [[pmin[i], pmax[i]] for i in range(n)]
    else:
        verts = [[tuple(f(v) for v in p[4 * k:4 * k + 3]) for k in range(3)] for p in prims]
        cent = []
        for vs in verts:
            bmn = [f(F32MAX)] * 3
            bmx = [f(-F32MAX)] * 3
            for v in vs:
                bmn = [lmin(bmn[k], v[k]) for k in range(3)]
            for v in vs:
                bmx = [lmax(bmx[k], v[k]) for k in range(3)]
            cent.append(tuple(f(bmn[k] + f(f(0.5) * f(bmx[k] - bmn[k]))) for k in range(3)))
        grow_pts = verts
    idx = list(range(n))

    def node_box(first, count):
        mn = [f(F32MAX)] * 3
        mx = [f(-F32MAX)] * 3
        for t in idx[first:first + count]:
            if tlas:
                mn = [lmin(mn[k], pmin[t][k]) for k in range(3)]
                mx = [lmax(mx[k], pmax[t][k]) for k in range(3)]
            else:
                for v in grow_pts[t]:
                    mn = [lmin(mn[k], v[k]) for k in range(3)]
                for v in grow_pts[t]:
                    mx = [lmax(mx[k], v[k]) for k in range(3)]
        return mn, mx

    def area(mn, mx):
        e = [f(mx[k] - mn[k]) for k in range(3)]
        return f(f(f(e[0] * e[1]) + f(e[1] * e[2])) + f(e[2] * e[0]))

    nodes = [[*node_box(0, n), 0, n]]

    def best_split(first, count):
        best = (0, f(0.0), f(1e30))
        for axis in range(3):
            bmin, bmax = f(1e30), f(-1e30)
            for t in idx[first:first + count]:
                bmin = lmin(bmin, cent[t][axis])
                bmax = lmax(bmax, cent[t][axis])
            if bmin == bmax:
                continue
            bb = [[[f(0)] * 3, [f(0)] * 3] for _ in range(bins)]
            bc = [0] * bins
            inv = f(f(bins) / f(bmax - bmin))
            for t in idx[first:first + count]:
                v = f(f(cent[t][axis] - bmin) * inv)
                b = 0 if not (v > 0) else min(bins - 1, int(v) if v < 2 ** 31 else bins - 1)
                bc[b] += 1
                for p in grow_pts[t]:
                    bb[b][0] = [lmin(bb[b][0][k], p[k]) for k in range(3)]
                    bb[b][1] = [lmax(bb[b][1][k], p[k]) for k in range(3)]
            ba = [[f(0)] * 3, [f(0)] * 3]
            bbx = [[f(0)] * 3, [f(0)] * 3]
            ca, cb = [0] * (bins - 1), [0] * (bins - 1)
            aa, ab = [f(0)] * (bins - 1), [f(0)] * (bins - 1)
            sa = sb = 0
            for i in range(bins - 1):
                sa += bc[i]
                ca[i] = sa
                for p in bb[i]:
                    ba = [[lmin(ba[0][k], p[k]) for k in range(3)], [lmax(ba[1][k], p[k]) for k in range(3)]]
                aa[i] = area(*ba)
                sb += bc[bins - 1 - i]
                cb[bins - 2 - i] = sb
                for p in bb[bins - 1 - i]:
                    bbx = [[lmin(bbx[0][k], p[k]) for k in range(3)], [lmax(bbx[1][k], p[k]) for k in range(3)]]
                ab[bins - 2 - i] = area(*bbx)
            size = f(f(bmax - bmin) / f(bins))
            for i in range(bins - 1):
                cost = f(f(f(ca[i]) * aa[i]) + f(f(cb[i]) * ab[i]))
                if cost < best[2]:
                    best = (axis, f(bmin + f(size * f(i + 1))), cost)
        return best

    stack = [0]
    while stack:
        ni = stack.pop()
        first, count = nodes[ni][2], nodes[ni][3]
        if count <= max_leaf:
            continue
        axis, pos, _ = best_split(first, count)
        i, j = first, first + count - 1
        while i <= j:
            if cent[idx[i]][axis] < pos:
                i += 1
            else:
                idx[i], idx[j] = idx[j], idx[i]
                j -= 1
        ac = i - first
        if ac == 0 or ac == count:
            continue
        ci = len(nodes)
        nodes.append([*node_box(first, ac), first, ac])
        nodes.append([*node_box(i, count - ac), i, count - ac])
        nodes[ni][2], nodes[ni][3] = ci, 0
        stack += [ci + 1, ci]
    out = np.zeros((len(nodes), 8), np.uint32)
    for k, (mn, mx, a, c) in enumerate(nodes):
        out[k, 0:3] = np.array(mn, np.float32).view(np.uint32)
        out[k, 3] = a
        out[k, 4:7] = np.array(mx, np.float32).view(np.uint32)
        out[k, 7] = c
    return out, np.array(idx, np.uint32)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("bins,leaf", [(20, 8), (16, 4), (4, 1), (32, 4)])
def test_blas_matches_literal_restatement(seed, bins, leaf):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(9, 120))
    c = rng.normal(size=(n, 1, 3)) * rng.uniform(0.5, 5.0)
    v = (c + rng.normal(size=(n, 3, 3)) * 0.3).astype(np.float32)
    if seed % 3 == 0:
        v[: n // 3] = np.round(v[: n // 3])  # coincident centroids on some axes
    prims = np.zeros((n, 12), np.float32)
    for k in range(3):
        prims[:, 4 * k:4 * k + 3] = v[:, k]
    nodes, idx = oracle.build_blas(prims, bins, leaf)
    pn, pi = py_build(prims, bins, leaf)
    assert np.array_equal(idx, pi)
    assert np.array_equal(nodes, pn)
    assert sorted(idx.tolist()) == list(range(n))


@pytest.mark.parametrize("seed", range(4))
def test_tlas_matches_literal_restatement(seed):
    rng = np.random.default_rng(100 + seed)
    k = int(rng.integers(2, 70))
    lo = rng.uniform(-10, 10, (k, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0.1, 3, (k, 3))).astype(np.float32)
    ce = (lo + np.float32(0.5) * (hi - lo)).astype(np.float32)
    b = np.concatenate([lo, hi, ce], 1)
    nodes, idx = oracle.build_tlas(b, 2, 1)
    pn, pi = py_build(None, 2, 1, tlas_bounds=b)
    assert np.array_equal(idx, pi)
    assert np.array_equal(nodes, pn)


def test_tlas_empty_scene_invalid_root():
    nodes, idx = oracle.build_tlas(np.zeros((0, 9), np.float32))
    assert nodes.shape == (1, 8) and not nodes.any() and idx.size == 0


def test_blas_degenerate_underflow_reported():
    # All centroids identical: every axis is skipped, split (axis 0, 0.0); all
    # centroids x >= 0 at first index 0 -> the reference's j underflows (panic).
    prims = np.zeros((12, 12), np.float32)
    prims[:, 4] = 1.0
    prims[:, 9] = 1.0
    with pytest.raises(RuntimeError, match="-7"):
        oracle.build_blas(prims, 20, 8)
    prims[:, 0:11:4] -= 5.0  # all centroids x < 0 -> no split, a single leaf
    nodes, idx = oracle.build_blas(prims, 20, 8)
    assert nodes.shape[0] == 1
