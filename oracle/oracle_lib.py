"""ORACLE TEST INFRASTRUCTURE — not part of the product.

ctypes access to oracle/liboracle.so, the CPU restatement of the hot path
(oracle/dspbr_oracle.cpp).  Used only by tests/, the smoke check and
bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_U = C.POINTER(C.c_uint32)
_D = C.POINTER(C.c_double)
_Q = C.POINTER(C.c_uint64)


class Params(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("fov", C.c_float), ("near_plane", C.c_float), ("width", C.c_int),
                ("height", C.c_int), ("max_bounces", C.c_int), ("use_ibl", C.c_int), ("bg_from_ibl", C.c_int),
                ("rr_start", C.c_int), ("env_mode", C.c_int), ("lean", C.c_int), ("pcg", C.c_int),
                ("ibl_rot_deg", C.c_float), ("bg", C.c_float * 4), ("ray_eps", C.c_float), ("clamp", C.c_float),
                ("rr_prob", C.c_float), ("seed", C.c_uint64), ("pl_pos", C.c_float * 4), ("pl_emis", C.c_float * 4)]


def build() -> str:
    src = os.path.join(HERE, "dspbr_oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def make_params(matrix, fov, near, width, height, max_bounces=8, use_ibl=1, bg_from_ibl=1, rr_start=2, env_mode=1,
                lean=0, pcg=0, ibl_rot_deg=0.0, bg=(0, 0, 0, 1), ray_eps=1e-4, clamp=3.0, rr_prob=0.1, seed=0,
                point_light=None):
    p = Params()
    for i, x in enumerate(np.asarray(matrix, np.float32).reshape(16)):
        p.view[i] = float(x)
    p.fov, p.near_plane, p.width, p.height = fov, near, width, height
    p.max_bounces, p.use_ibl, p.bg_from_ibl, p.rr_start = max_bounces, use_ibl, bg_from_ibl, rr_start
    p.env_mode, p.lean, p.pcg, p.ibl_rot_deg = env_mode, lean, pcg, ibl_rot_deg
    for i in range(4):
        p.bg[i] = bg[i]
    p.ray_eps, p.clamp, p.rr_prob, p.seed = ray_eps, clamp, rr_prob, seed
    if point_light is not None:  # ((x, y, z), (r, g, b))
        for i in range(3):
            p.pl_pos[i], p.pl_emis[i] = float(point_light[0][i]), float(point_light[1][i])
        p.pl_pos[3] = p.pl_emis[3] = 1.0
    return p


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(build())
        self._keep = []

    def set_scene(self, vertices, indices, materials, nodes, remap):
        v = np.ascontiguousarray(vertices, np.float32)
        i = np.ascontiguousarray(indices, np.uint32)
        m = np.ascontiguousarray(materials, np.float32)
        n = np.ascontiguousarray(nodes, np.float32)
        r = np.ascontiguousarray(remap, np.int32)
        self._keep = [v, i, m, n, r]
        rc = self.lib.orc_set_scene(v.ctypes.data_as(_F), v.size // 20, i.ctypes.data_as(_U), i.size,
                                    m.ctypes.data_as(_F), m.size // 68, n.ctypes.data_as(_F), n.size // 16,
                                    r.ctypes.data_as(_I), r.size)
        if rc != 0:
            raise ValueError("oracle rejected the scene")

    def set_ibl(self, rgba):
        img = np.ascontiguousarray(rgba, np.float32)
        self.env_w, self.env_h = img.shape[1], img.shape[0]
        self.lib.orc_set_ibl(img.ctypes.data_as(_F), img.shape[1], img.shape[0])

    def ibl_tables(self):
        n = self.env_w * self.env_h
        pdf, cdf = np.zeros(n, np.float32), np.zeros(n, np.float32)
        ypdf, ycdf = np.zeros(self.env_h, np.float32), np.zeros(self.env_h, np.float32)
        prob, alias = np.zeros(n, np.float32), np.zeros(n, np.int32)
        tot = C.c_double()
        self.lib.orc_get_ibl_tables(pdf.ctypes.data_as(_F), cdf.ctypes.data_as(_F), ypdf.ctypes.data_as(_F),
                                    ycdf.ctypes.data_as(_F), C.byref(tot), prob.ctypes.data_as(_F),
                                    alias.ctypes.data_as(_I))
        return {"pdf": pdf, "cdf": cdf, "yPdf": ypdf, "yCdf": ycdf, "totalSum": tot.value, "aliasProb": prob,
                "alias": alias}

    def trace(self, rays8, mode=0):
        """mode 0: BVH closest hit, 1: brute force, 2: isOccluded.  Returns tri, t, uv, counters."""
        r = np.ascontiguousarray(rays8, np.float32)
        n = r.shape[0]
        tri, t, uv = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32)
        cnt = np.zeros(4, np.uint64)
        self.lib.orc_f32_trace(n, r.ctypes.data_as(_F), mode, tri.ctypes.data_as(_I), t.ctypes.data_as(_F),
                               uv.ctypes.data_as(_F), cnt.ctypes.data_as(_Q))
        return tri, t, uv, {"rays": int(cnt[0]), "nodes": int(cnt[1]), "tris": int(cnt[2]), "aborted": int(cnt[3])}

    def brute_force64(self, rays8):
        r = np.ascontiguousarray(rays8, np.float32)
        n = r.shape[0]
        tri, t = np.zeros(n, np.int32), np.zeros(n, np.float64)
        self.lib.orc_f64_brute_force(n, r.ctypes.data_as(_F), tri.ctypes.data_as(_I), t.ctypes.data_as(_D))
        return tri, t

    def bsdf(self, hit20, wo3, rnd4, precision="f32", lean=0):
        h = np.ascontiguousarray(hit20, np.float32)
        w = np.ascontiguousarray(wo3, np.float32)
        r = np.ascontiguousarray(rnd4, np.float32)
        n = h.shape[0]
        ev, sm, fl = np.zeros((n, 4), np.float32), np.zeros((n, 10), np.float32), np.zeros(n, np.int32)
        fn = self.lib.orc_f32_bsdf if precision == "f32" else self.lib.orc_f64_bsdf
        fn(n, h.ctypes.data_as(_F), w.ctypes.data_as(_F), r.ctypes.data_as(_F), lean, ev.ctypes.data_as(_F),
           sm.ctypes.data_as(_F), fl.ctypes.data_as(_I))
        return ev, sm, fl

    def ibl(self, r2, dirs3, rot_deg=0.0, mode=1):
        r = np.ascontiguousarray(r2, np.float32)
        d = np.ascontiguousarray(dirs3, np.float32)
        n = r.shape[0]
        sdp, pdf, rgb = np.zeros((n, 4), np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        self.lib.orc_f32_ibl(n, r.ctypes.data_as(_F), d.ctypes.data_as(_F), C.c_float(rot_deg), mode,
                             sdp.ctypes.data_as(_F), pdf.ctypes.data_as(_F), rgb.ctypes.data_as(_F))
        return sdp, pdf, rgb

    def camera_rays(self, params, xy, r2):
        xy = np.ascontiguousarray(xy, np.int32)
        r2 = np.ascontiguousarray(r2, np.float32)
        out = np.zeros((xy.shape[0], 6), np.float32)
        self.lib.orc_f32_camera_rays(C.byref(params), xy.shape[0], xy.ctypes.data_as(_I), r2.ctypes.data_as(_F),
                                     out.ctypes.data_as(_F))
        return out

    def rng(self, n, x=0, y=0, mwc_seed=0, pcg=False, seed=0, stream=0):
        out = np.zeros(n, np.float32)
        self.lib.orc_rng(int(pcg), C.c_uint64(seed), C.c_uint64(stream), x, y, mwc_seed, n, out.ctypes.data_as(_F))
        return out

    def render(self, params, xy, frame, precision="f32", threads=0):
        """One sample per listed pixel at progressive frame `frame`; returns (rgba, counters)."""
        threads = threads or (os.cpu_count() or 1)
        xy = np.ascontiguousarray(xy, np.int32)
        out = np.zeros((xy.shape[0], 4), np.float32)
        cnt = np.zeros(4, np.uint64)
        fn = self.lib.orc_f32_render if precision == "f32" else self.lib.orc_f64_render
        fn(C.byref(params), xy.shape[0], xy.ctypes.data_as(_I), C.c_uint32(frame), out.ctypes.data_as(_F), threads,
           cnt.ctypes.data_as(_Q))
        return out, {"rays": int(cnt[0]), "nodes": int(cnt[1]), "tris": int(cnt[2]), "aborted": int(cnt[3])}

    def render_image(self, params, frames, precision="f32", first_frame=1):
        """Running mean over `frames` progressive frames of the full image, (H, W, 4)."""
        W, H = params.width, params.height
        ys, xs = np.mgrid[0:H, 0:W]
        xy = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
        acc = np.zeros((H * W, 4), np.float64)
        for f in range(first_frame, first_frame + frames):
            out, _ = self.render(params, xy, f, precision)
            acc += out
        return (acc / frames).reshape(H, W, 4).astype(np.float32)


def all_pixels(width, height):
    ys, xs = np.mgrid[0:height, 0:width]
    return np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
