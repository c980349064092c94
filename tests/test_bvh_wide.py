"""The 4-wide BVH the path kernels traverse (DSPBR_TRAVERSAL_WIDE), on the CPU.

dspbr_bvh_wide collapses a reference-layout binary BVH; a float32 model of the
device's wide traversal (same slab and Moller-Trumbore arithmetic, children
visited near to far) must find the same closest t as the oracle's restatement
of the reference's binary traversal (bvh.glsl:149-212), and the same triangle
except where two triangles hit at exactly that t.
"""
import ctypes as C

import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh
from oracle import oracle_lib
from tests import helpers

F = np.float32
FAR = F(1e30)


def collapse(bvh: Bvh):
    lib = _lib.load()
    nodes = np.ascontiguousarray(bvh.nodes, np.float32)
    nn, nl, root = C.c_uint32(), C.c_uint32(), C.c_int32()
    n_nodes = nodes.size // 16
    assert lib.dspbr_bvh_wide(_lib.fptr(nodes), n_nodes, bvh.indices.size, C.byref(nn), C.byref(nl), C.byref(root),
                              None, None) == 0
    w = np.zeros(nn.value * 32, np.float32)
    lv = np.zeros(max(nl.value, 1) * 2, np.int32)
    assert lib.dspbr_bvh_wide(_lib.fptr(nodes), n_nodes, bvh.indices.size, None, None, None, _lib.fptr(w),
                              _lib.iptr(lv)) == 0
    w = w.reshape(-1, 32)
    boxes = w[:, :24].reshape(-1, 6, 4)           # lo_x, lo_y, lo_z, hi_x, hi_y, hi_z  x 4 children
    ints = w[:, 24:].copy().view(np.int32)        # child[4], count, pad[3]
    return boxes, ints[:, :4], ints[:, 4], lv.reshape(-1, 2)[: nl.value], root.value


def slab(lo, hi, o, inv, tfar):
    t0 = [(F(lo[a]) - o[a]) * inv[a] for a in range(3)]
    t1 = [(F(hi[a]) - o[a]) * inv[a] for a in range(3)]
    mn = lambda x, y: y if y < x else x
    mx = lambda x, y: y if x < y else x
    tmin = mx(mx(mn(t0[0], t1[0]), mn(t0[1], t1[1])), mn(t0[2], t1[2]))
    tmax = mn(mn(mx(t0[0], t1[0]), mx(t0[1], t1[1])), mx(t0[2], t1[2]))
    if tmin > tmax or tmax < 0 or tmin >= tfar:
        return FAR
    return tmin


def cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], F)


def dot(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


def intersect(o, d, p0, e0, e1, tfar):
    pv = cross(d, e1)
    det = dot(e0, pv)
    if abs(det) < F(1e-8):
        return None
    f = F(1) / det
    s = (o - p0).astype(F)
    u = f * dot(s, pv)
    if u < 0 or u > 1:
        return None
    q = cross(s, e0)
    v = f * dot(d, q)
    if v < 0 or u + v > 1:
        return None
    t = f * dot(e1, q)
    if t < F(1e-8) or t >= tfar:
        return None
    return t


def trace_wide(w, tris, o, d, tfar):
    boxes, child, count, leaves, root = w
    inv = np.array([F(1) / d[0], F(1) / d[1], F(1) / d[2]], F)
    best_t, best = F(tfar), -1
    stack = [root]
    while stack:
        e = stack.pop()
        if e < 0:
            b, en = leaves[~e]
            for i in range(b, en):
                tid, p0, e0, e1 = tris[i]
                if tid < 0:
                    continue
                t = intersect(o, d, p0, e0, e1, best_t)
                if t is not None:
                    best_t, best = t, tid
            continue
        hits = []
        for k in range(count[e]):
            lo = boxes[e, 0:3, k]
            hi = boxes[e, 3:6, k]
            dk = slab(lo, hi, o, inv, best_t)
            if dk < FAR:
                hits.append((dk, k))
        for dk, k in sorted(hits, reverse=True):
            stack.append(int(child[e, k]))
    return best, best_t


def leaf_tris(sc, bvh):
    v = sc.vertices.reshape(-1, 20)[:, :3].astype(F)
    idx = sc.indices.reshape(-1, 3)
    out = []
    for t in bvh.indices:
        if t < 0 or t >= idx.shape[0]:
            out.append((-1, None, None, None))
            continue
        p0, p1, p2 = v[idx[t, 0]], v[idx[t, 1]], v[idx[t, 2]]
        out.append((int(t), p0, (p1 - p0).astype(F), (p2 - p0).astype(F)))
    return out


@pytest.mark.parametrize("which", ["small", "sized"])
def test_wide_collapse_same_closest_hits(which):
    sc = synth.make_small(0) if which == "small" else synth.make_sized(4, 6000, env_size=(32, 16))
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    w = collapse(bvh)
    boxes, child, count, leaves, root = w
    n_bin = bvh.nodes.size // 16
    assert root == 0 and 1 <= count.min() and count.max() <= 4
    assert len(boxes) < 0.5 * n_bin  # about a third of the binary node count
    # every binary leaf becomes exactly one wide leaf covering its slots
    covered = np.zeros(bvh.indices.size, np.int32)
    for b, e in leaves:
        covered[b:e] += 1
    assert (covered == 1).all()
    tris = leaf_tris(sc, bvh)
    o = oracle_lib.Oracle()
    o.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    rays = helpers.random_rays(sc.vertices, 300, seed=31)
    ref_tri, ref_t, _, stats = o.trace(rays, mode=0)
    assert stats["aborted"] == 0
    ties = 0
    for r in range(rays.shape[0]):
        tri, t = trace_wide(w, tris, rays[r, 0:3].astype(F), rays[r, 3:6].astype(F), F(rays[r, 6]))
        assert tri >= 0 or ref_tri[r] < 0
        if ref_tri[r] < 0:
            assert tri < 0
            continue
        assert np.float32(t).view(np.int32) == ref_t[r].view(np.int32), r
        ties += int(tri != ref_tri[r])
    assert ties <= 3


def test_wide_root_leaf_and_malformed_children():
    # a single-leaf BVH: the root is a leaf (tested without a box)
    nodes = np.zeros(16, np.float32)
    nodes[11], nodes[15] = 2, 0  # cnt = 2, first = 0
    lib = _lib.load()
    nn, nl, root = C.c_uint32(), C.c_uint32(), C.c_int32()
    assert lib.dspbr_bvh_wide(_lib.fptr(nodes), 1, 2, C.byref(nn), C.byref(nl), C.byref(root), None, None) == 0
    assert (nn.value, nl.value, root.value) == (0, 1, -1)
    # an inner root whose children are out of range or itself: nothing pushed
    nodes = np.zeros(16, np.float32)
    nodes[3], nodes[7] = 5, 0  # left = 5 (out of range), right = 0 (self)
    assert lib.dspbr_bvh_wide(_lib.fptr(nodes), 1, 0, C.byref(nn), C.byref(nl), C.byref(root), None, None) == 0
    w = np.zeros(32, np.float32)
    lib.dspbr_bvh_wide(_lib.fptr(nodes), 1, 0, None, None, None, _lib.fptr(w), None)
    assert nn.value == 1 and w[24:].view(np.int32)[4] == 0  # no children
