"""ORACLE TEST INFRASTRUCTURE — not part of the product.

ctypes access to oracle/_ref/libglslref_{f32,f64}.so: the reference's own
fragment shader (packages/lib/shader/**, compiled as C++ by
oracle/ref/build_ref.sh) driven by a host harness that plays WebGL2's role.
Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_U = C.POINTER(C.c_uint32)
_D = C.POINTER(C.c_double)


def available(precision: str = "f32") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libglslref_{precision}.so"))


def _f(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(_F)


class GlslReference:
    """The reference shader compiled for the host, FP32 ('f32') or FP64 ('f64')."""

    def __init__(self, precision: str = "f32"):
        path = os.path.join(REF_DIR, f"libglslref_{precision}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (oracle/ref/build_ref.sh)")
        self.lib = C.CDLL(path)
        self.p = f"ref_{precision}_"
        self._keep = []

    def fn(self, name):
        return getattr(self.lib, self.p + name)

    def set_scene(self, vertices, indices, materials, nodes, remap):
        v = np.ascontiguousarray(vertices, np.float32)
        i = np.ascontiguousarray(indices, np.uint32)
        m = np.ascontiguousarray(materials, np.float32)
        n = np.ascontiguousarray(nodes, np.float32)
        r = np.ascontiguousarray(remap, np.int32)
        self._keep = [v, i, m, n, r]
        rc = self.fn("set_scene")(v.ctypes.data_as(_F), v.size // 20, i.ctypes.data_as(_U), i.size,
                                  m.ctypes.data_as(_F), m.size // 68, n.ctypes.data_as(_F), n.size // 16,
                                  r.ctypes.data_as(_I), r.size)
        if rc != 0:
            raise ValueError("reference harness rejected the scene")

    def set_textures(self, infos, arrays):
        """infos: (N, 8) TexInfo records; arrays: list of uint8 (layers, h, w, 4) texture arrays."""
        inf = np.ascontiguousarray(infos, np.float32).reshape(-1, 8)
        arrs = [np.ascontiguousarray(a, np.uint8) for a in arrays]
        ptrs = (C.c_void_p * max(len(arrs), 1))(*[a.ctypes.data for a in arrs])
        whl = np.array([[a.shape[2], a.shape[1], a.shape[0]] for a in arrs] or [[0, 0, 0]], np.int32).reshape(-1)
        self._tex_keep = [inf, arrs, ptrs, whl]
        fn = self.fn("set_textures")
        fn.argtypes = [_F, C.c_int, C.c_int, C.POINTER(C.c_void_p), _I]
        if fn(inf.ctypes.data_as(_F), inf.shape[0], len(arrs), ptrs, whl.ctypes.data_as(_I)) != 0:
            raise ValueError("reference harness rejected the textures")

    def set_ibl(self, rgba):
        img = np.ascontiguousarray(rgba, np.float32)
        self._env = img
        self.env_w, self.env_h = img.shape[1], img.shape[0]
        if self.fn("set_ibl")(img.ctypes.data_as(_F), img.shape[1], img.shape[0]) != 0:
            raise ValueError("reference harness rejected the environment map")

    def ibl_tables(self):
        n = self.env_w * self.env_h
        pdf, cdf = np.zeros(n, np.float32), np.zeros(n, np.float32)
        ypdf, ycdf = np.zeros(self.env_h, np.float32), np.zeros(self.env_h, np.float32)
        tot = C.c_double()
        self.fn("get_ibl_tables")(pdf.ctypes.data_as(_F), cdf.ctypes.data_as(_F), ypdf.ctypes.data_as(_F),
                                  ycdf.ctypes.data_as(_F), C.byref(tot))
        return {"pdf": pdf, "cdf": cdf, "yPdf": ypdf, "yCdf": ycdf, "totalSum": tot.value}

    def set_uniforms(self, block: np.ndarray):
        b = np.ascontiguousarray(block, np.float32)
        assert b.size == 52
        self.fn("set_uniforms")(b.ctypes.data_as(_F))

    def render(self, width, height, accum: np.ndarray, threads: int = 0) -> np.ndarray:
        threads = threads or (os.cpu_count() or 1)
        assert accum.dtype == np.float32 and accum.flags.c_contiguous and accum.shape == (height, width, 4)
        rc = self.fn("render")(width, height, accum.ctypes.data_as(_F), threads)
        if rc != 0:
            raise ValueError("reference render failed (a texture id beyond the TexInfo table)")
        return accum

    def render_pixels(self, xy, width, height, threads: int = 0):
        """One frame (frame number from the uniform block) of the listed pixels; returns (rgba, rays traced)."""
        threads = threads or (os.cpu_count() or 1)
        xy = np.ascontiguousarray(xy, np.int32)
        out = np.zeros((xy.shape[0], 4), np.float32)
        rays = C.c_uint64()
        self.fn("render_pixels")(xy.shape[0], xy.ctypes.data_as(_I), width, height, out.ctypes.data_as(_F), threads,
                                 C.byref(rays))
        return out, rays.value

    def trace(self, rays8: np.ndarray):
        r = np.ascontiguousarray(rays8, np.float32)
        n = r.shape[0]
        tri, t, uv = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32)
        self.fn("trace")(n, r.ctypes.data_as(_F), tri.ctypes.data_as(_I), t.ctypes.data_as(_F),
                         uv.ctypes.data_as(_F))
        return tri, t, uv

    def occluded(self, rays8: np.ndarray):
        r = np.ascontiguousarray(rays8, np.float32)
        occ = np.zeros(r.shape[0], np.int32)
        self.fn("occluded")(r.shape[0], r.ctypes.data_as(_F), occ.ctypes.data_as(_I))
        return occ

    def camera_rays(self, xy, r2, width, height):
        xy = np.ascontiguousarray(xy, np.int32)
        r2 = np.ascontiguousarray(r2, np.float32)
        out = np.zeros((xy.shape[0], 6), np.float32)
        self.fn("camera_ray")(xy.shape[0], xy.ctypes.data_as(_I), r2.ctypes.data_as(_F), width, height,
                              out.ctypes.data_as(_F))
        return out

    def rng(self, x, y, seed, n):
        out = np.zeros(n, np.float32)
        self.fn("rng")(x, y, seed, n, out.ctypes.data_as(_F))
        return out

    def bsdf(self, hit20, wo3, rnd4):
        h = np.ascontiguousarray(hit20, np.float32)
        w = np.ascontiguousarray(wo3, np.float32)
        r = np.ascontiguousarray(rnd4, np.float32)
        n = h.shape[0]
        ev, sm, fl = np.zeros((n, 4), np.float32), np.zeros((n, 10), np.float32), np.zeros(n, np.int32)
        self.fn("bsdf")(n, h.ctypes.data_as(_F), w.ctypes.data_as(_F), r.ctypes.data_as(_F),
                        ev.ctypes.data_as(_F), sm.ctypes.data_as(_F), fl.ctypes.data_as(_I))
        return ev, sm, fl

    def ibl(self, r2, dirs3):
        r = np.ascontiguousarray(r2, np.float32)
        d = np.ascontiguousarray(dirs3, np.float32)
        n = r.shape[0]
        sdp, pdf, rgb = np.zeros((n, 4), np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        self.fn("ibl")(n, r.ctypes.data_as(_F), d.ctypes.data_as(_F), sdp.ctypes.data_as(_F),
                       pdf.ctypes.data_as(_F), rgb.ctypes.data_as(_F))
        return sdp, pdf, rgb

    def tonemap(self, rgba, exposure: float, gamma: bool, mode: int) -> np.ndarray:
        """tonemap.frag over an (H, W, 4) RGBA32F image (renderer.ts:668-676)."""
        img = np.ascontiguousarray(rgba, np.float32)
        out = np.zeros_like(img)
        fn = self.fn("tonemap")
        fn.argtypes = [_F, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, _F]
        fn(img.ctypes.data_as(_F), img.shape[1], img.shape[0], float(exposure), int(bool(gamma)), int(mode),
           out.ctypes.data_as(_F))
        return out

    def fxaa(self, rgba) -> np.ndarray:
        """fxaa.frag over an (H, W, 4) RGBA32F image (renderer.ts:678-686)."""
        img = np.ascontiguousarray(rgba, np.float32)
        out = np.zeros_like(img)
        fn = self.fn("fxaa")
        fn.argtypes = [_F, C.c_int, C.c_int, _F]
        fn(img.ctypes.data_as(_F), img.shape[1], img.shape[0], out.ctypes.data_as(_F))
        return out


def uniform_block(camera_matrix, fov_deg, near, width, height, frame, max_bounces, use_ibl=1, ibl_rotation=0.0,
                  background_from_ibl=1, background_color=(0, 0, 0, 1), ray_eps=1e-4, clamp_threshold=3.0,
                  point_light=None):
    """The std140 uniform block as renderer.ts:376-449 fills it (52 floats)."""
    b = np.zeros(52, np.float32)
    m = np.asarray(camera_matrix, np.float32).reshape(16)
    b[0:16] = m
    b[16:20] = background_color
    film = np.tan(np.float64(fov_deg) * 0.5 * np.pi / 180.0) * np.float64(near)
    b[20:23] = m[12:15]
    b[23] = film
    b[24:26] = [1.0 / width, 1.0 / height]
    b[28] = frame
    b[31] = use_ibl
    b[32] = np.float64(ibl_rotation) / 180.0 * np.pi
    b[33] = background_from_ibl
    b[34] = max_bounces
    b[35] = near
    b[37] = ray_eps
    b[38] = clamp_threshold
    if point_light is not None:
        b[44:47] = point_light[0]
        b[47] = 1
        b[48:51] = point_light[1]
        b[51] = 1
    return b
