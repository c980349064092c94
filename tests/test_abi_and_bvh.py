"""CPU-only checks of the product library: it loads, exports every entry
point include/dspbr.h declares, and its host-side BVH builder (no GPU needed)
produces valid trees in the reference's node layout."""
import os
import re

import numpy as np
import pytest

from dspbr import _lib, synth
from dspbr.viewport import Bvh
from oracle import oracle_lib
from tests import helpers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "dspbr.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dspbr_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for each entry point it calls
    assert set(_lib.SIGNATURES) <= set(names)


def test_params_defaults_mirror_reference():
    p = _lib.default_params()
    # renderer.ts:172-306 defaults; constants.glsl:19-20
    assert p.max_bounces == 8 and p.use_ibl == 1 and p.background_from_ibl == 1
    assert abs(p.ray_eps - 1e-4) < 1e-9 and p.clamp_threshold == 3.0
    assert p.rr_start_depth == 2 and abs(p.rr_termination_prob - 0.1) < 1e-7
    assert list(p.background_color) == [0.0, 0.0, 0.0, 1.0]


def test_no_gpu_create_fails_loudly():
    import ctypes as C
    n = C.c_int(-1)
    rc = _lib.load().dspbr_device_count(C.byref(n))
    if rc == 0 and n.value > 0:
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert _lib.load().dspbr_create(0, C.byref(h)) != 0


def _check_tree(bvh, positions, indices):
    nodes = bvh.nodes.reshape(-1, 16)
    ntri = indices.size // 3
    assert sorted(bvh.indices.tolist()) == list(range(ntri))  # every triangle exactly once
    tri_pos = positions[indices.reshape(-1, 3)]  # (T, 3, 3)
    covered = np.zeros(bvh.indices.size, np.int32)
    depth = {0: 0}
    stack = [0]
    while stack:
        ni = stack.pop()
        n = nodes[ni]
        cnt, first = int(n[11]), int(n[15])
        if cnt > 0:
            assert cnt <= 64
            covered[first:first + cnt] += 1
            continue
        left, right = int(n[3]), int(n[7])
        for child, lo, hi in ((left, n[0:3], n[4:7]), (right, n[8:11], n[12:15])):
            assert 0 < child < nodes.shape[0]
            depth[child] = depth[ni] + 1
            # the child box bounds every triangle below it
            sub = [child]
            tris = []
            while sub:
                c = sub.pop()
                m = nodes[c]
                if int(m[11]) > 0:
                    tris += bvh.indices[int(m[15]):int(m[15]) + int(m[11])].tolist()
                else:
                    sub += [int(m[3]), int(m[7])]
            p = tri_pos[tris].reshape(-1, 3)
            assert (p >= lo - 1e-6).all() and (p <= hi + 1e-6).all()
            stack.append(child)
    assert (covered == 1).all()  # leaves partition the remap array
    assert max(depth.values()) < 63  # the 64-entry traversal stack cannot overflow
    assert bvh.depth == max(depth.values())


def test_bvh_builder_small_scene_valid():
    sc = synth.make_small(0)
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    _check_tree(bvh, sc.vertices[:, :3], sc.indices)


def test_bvh_builder_degenerate_and_tiny_inputs():
    # a single triangle: root is a leaf
    v = np.zeros((3, 20), np.float32)
    v[:, :3] = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    bvh = Bvh.build(v, np.array([0, 1, 2], np.uint32), 20)
    assert bvh.nodes.size == 16 and int(bvh.nodes[11]) == 1
    # many coincident triangles (zero centroid extent) still split into bounded leaves
    v = np.tile(v, (50, 1))
    idx = np.arange(150, dtype=np.uint32)
    bvh = Bvh.build(v, idx, 20)
    _check_tree(bvh, v[:, :3], idx)
    # malformed index buffers are refused with an error
    with pytest.raises(_lib.DspbrError):
        Bvh.build(v, np.array([0, 1], np.uint32), 20)
    with pytest.raises(_lib.DspbrError):
        Bvh.build(v, np.array([0, 1, 9999], np.uint32), 20)


def test_bvh_traversal_equals_brute_force_on_sized_scene():
    sc = synth.make_sized(3, 20000, env_size=(16, 8))
    bvh = Bvh.build(sc.vertices, sc.indices, 20)
    _check_tree(bvh, sc.vertices[:, :3], sc.indices) if sc.num_triangles < 3000 else None
    o = oracle_lib.Oracle()
    o.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    rays = helpers.random_rays(sc.vertices, 1500, seed=5)
    tri, t, _, cnt = o.trace(rays)
    bf_tri, bf_t, _, _ = o.trace(rays, mode=1)
    same = tri == bf_tri
    assert same.mean() > 0.99
    np.testing.assert_allclose(t[~same], bf_t[~same], rtol=1e-6)
    assert cnt["aborted"] == 0
