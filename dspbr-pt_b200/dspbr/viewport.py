"""Host-side mirror of the reference's embedding API.

`PathtracingViewport` keeps the method names, argument meaning and error
behaviour of packages/lib/pathtracing_viewport.ts:100-342 (settings, setScene,
setIBL, setCamera / setLookAtCamera, resize, start / stop, resetAccumulation,
diagnostics, events).  Rendering goes through the C ABI of libdspbr_cuda.so;
the WebGL canvas becomes a headless device buffer read back with
readAccumulation().  Display-only settings (tone mapping, exposure, gamma,
FXAA, pixel ratio, tiling) are accepted and stored: they act after the
accumulation buffer, outside the path-tracing hot path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, f32, fptr, iptr, uptr
from .synth import MATERIAL_STRIDE, VERTEX_STRIDE


class Bvh:
    """BVH in the reference's node layout (replaces buildIndexedBvh, tinybvh_builder.ts:142-215)."""

    def __init__(self, nodes: np.ndarray, indices: np.ndarray, depth: int, triangles: int):
        self.nodes = nodes
        self.indices = indices
        self.depth = depth
        self.triangles = triangles

    @staticmethod
    def build(positions: np.ndarray, indices: np.ndarray, stride: int | None = None) -> "Bvh":
        lib = _lib.load()
        pos = f32(positions)
        if stride is None:
            stride = pos.shape[1] if pos.ndim == 2 else 3
        idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        h = C.c_void_p()
        rc = lib.dspbr_bvh_build(fptr(pos), pos.size // stride, stride, uptr(idx), idx.size, C.byref(h))
        try:
            if rc != 0:
                buf = C.create_string_buffer(256)
                if h:
                    lib.dspbr_bvh_error(h, buf, 256)
                raise _lib.DspbrError(rc, "BVH build failed: " + buf.value.decode())
            nn, ni, dep, nt = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
            lib.dspbr_bvh_info(h, C.byref(nn), C.byref(ni), C.byref(dep), C.byref(nt))
            nodes = np.zeros(nn.value * 16, np.float32)
            remap = np.zeros(ni.value, np.int32)
            check(lib.dspbr_bvh_copy(h, fptr(nodes), iptr(remap)))
            return Bvh(nodes, remap, dep.value, nt.value)
        finally:
            lib.dspbr_bvh_free(h)


class Context:
    """One CUDA device + stream (the C ABI's dspbr_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        check(self.lib.dspbr_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.dspbr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        check(rc, self.h)

    def set_bvh_builder(self, builder: str) -> None:
        """BVH builder of scenes created without one: "host" (binned SAH on the
        host), "device" (binned SAH on the device) or "device_lbvh" (linear
        BVH on the device: the fastest build)."""
        codes = {"host": _lib.BVH_BUILD_HOST, "device": _lib.BVH_BUILD_DEVICE,
                 "device_lbvh": _lib.BVH_BUILD_DEVICE_LBVH}
        if builder not in codes:
            raise ValueError(f"set_bvh_builder: {builder!r} is not one of {sorted(codes)}")
        self.check(self.lib.dspbr_set_bvh_builder(self.h, codes[builder]))

    def set_wide_bvh(self, width: int) -> None:
        """Width of the wide BVH the path kernels trace in scenes created
        afterwards: 4 (float boxes) or 8 (compressed: quantised child boxes)."""
        if width not in (4, 8):
            raise ValueError(f"set_wide_bvh: {width!r} is not 4 or 8")
        self.check(self.lib.dspbr_set_wide_bvh(self.h, int(width)))

    def host_array(self, shape, dtype=np.float32) -> np.ndarray:
        """numpy array over page-locked host memory (dspbr_host_alloc)."""
        import weakref
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = C.c_void_p()
        self.check(self.lib.dspbr_host_alloc(self.h, n, C.byref(p)))
        raw = (C.c_byte * n).from_address(p.value)
        # freed with the buffer, also after the context is closed
        weakref.finalize(raw, self.lib.dspbr_host_free, None, C.c_void_p(p.value))
        return np.frombuffer(raw, dtype=dtype).reshape(shape)


def apply_scene_lights(params, lights) -> bool:
    """The first scene light drives u_point_light_* whatever its type
    (renderer.ts:424-430); no light disables it (w = 0).  Returns whether the
    parameters changed."""
    pos, emis = (0.0, 0.0, 0.0, 0.0), (0.0, 0.0, 0.0, 0.0)
    if lights:
        pos = (*[float(x) for x in lights[0]["position"]], 1.0)
        emis = (*[float(x) for x in lights[0]["emission"]], 1.0)
    changed = tuple(params.point_light_position) != pos or tuple(params.point_light_emission) != emis
    for k in range(4):
        params.point_light_position[k] = pos[k]
        params.point_light_emission[k] = emis[k]
    return changed


class DeviceScene:
    """Scene resident on the device (dspbr_scene)."""

    def __init__(self, ctx: Context, vertices, indices, materials, bvh: Bvh | None = None, lights=None):
        self.ctx = ctx
        self.lights = list(lights or [])  # host-side: requests on this scene take their point light from it
        v = f32(vertices).reshape(-1, VERTEX_STRIDE)
        i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        m = f32(materials).reshape(-1, MATERIAL_STRIDE)
        h = C.c_void_p()
        if bvh is None:
            rc = ctx.lib.dspbr_scene_create(ctx.h, fptr(v), v.shape[0], uptr(i), i.size, fptr(m), m.shape[0],
                                            None, 0, None, 0, C.byref(h))
        else:
            rc = ctx.lib.dspbr_scene_create(ctx.h, fptr(v), v.shape[0], uptr(i), i.size, fptr(m), m.shape[0],
                                            fptr(bvh.nodes), bvh.nodes.size // 16, iptr(bvh.indices),
                                            bvh.indices.size, C.byref(h))
        ctx.check(rc)
        self.h = h
        self.num_triangles = i.size // 3

    def update_materials(self, materials, first: int = 0):
        m = f32(materials).reshape(-1, MATERIAL_STRIDE)
        self.ctx.check(self.ctx.lib.dspbr_scene_update_materials(self.h, fptr(m), first, m.shape[0]))

    def update_vertices(self, vertices, first: int = 0) -> None:
        """New 20-float records for vertices [first, first + n) (same triangles); the
        BVH is refitted on the device (dspbr_scene_update_vertices)."""
        v = f32(vertices).reshape(-1, VERTEX_STRIDE)
        self.ctx.check(self.ctx.lib.dspbr_scene_update_vertices(self.h, fptr(v), int(first), v.shape[0]))

    def set_textures(self, tex_infos, arrays) -> None:
        """Material textures: (N, 8) TexInfo records and RGBA8 arrays of shape
        (layers, height, width, 4) (dspbr_scene_set_textures)."""
        infos = f32(tex_infos).reshape(-1, 8)
        arrs = [np.ascontiguousarray(a, np.uint8) for a in arrays]
        desc = (_lib.TextureArray * max(len(arrs), 1))()
        for k, a in enumerate(arrs):
            desc[k].layers, desc[k].height, desc[k].width = a.shape[0], a.shape[1], a.shape[2]
            desc[k].rgba8 = a.ctypes.data
        self.ctx.check(self.ctx.lib.dspbr_scene_set_textures(self.h, fptr(infos), infos.shape[0], desc, len(arrs)))

    def bvh(self) -> "Bvh":
        """The scene's binary BVH in the reference layout, read back from the device."""
        nn, ni = C.c_uint32(), C.c_uint32()
        self.ctx.check(self.ctx.lib.dspbr_scene_bvh(self.h, None, None, C.byref(nn), C.byref(ni)))
        nodes = np.zeros(nn.value * 16, np.float32)
        remap = np.zeros(ni.value, np.int32)
        self.ctx.check(self.ctx.lib.dspbr_scene_bvh(self.h, fptr(nodes), iptr(remap), None, None))
        return Bvh(nodes, remap, 0, self.num_triangles)

    def wide_bvh(self) -> dict:
        """The wide BVH the path kernels use: width (4 or 8), nodes and, for
        the 8-wide tree, its depth in levels."""
        w, nodes, levels = C.c_int(), C.c_uint32(), C.c_uint32()
        self.ctx.check(self.ctx.lib.dspbr_scene_wide_bvh(self.h, C.byref(w), C.byref(nodes), C.byref(levels)))
        return {"width": w.value, "nodes": nodes.value, "levels": levels.value}

    def device_bytes(self) -> int:
        b = C.c_uint64()
        self.ctx.check(self.ctx.lib.dspbr_scene_device_bytes(self.h, C.byref(b)))
        return b.value

    def close(self):
        if self.h:
            self.ctx.lib.dspbr_scene_destroy(self.h)
            self.h = None


class DeviceIbl:
    """Environment map + importance tables on the device (dspbr_ibl)."""

    def __init__(self, ctx: Context, rgba: np.ndarray):
        self.ctx = ctx
        img = f32(rgba)
        self.height, self.width = img.shape[0], img.shape[1]
        h = C.c_void_p()
        ctx.check(ctx.lib.dspbr_ibl_create(ctx.h, fptr(img), self.width, self.height, C.byref(h)))
        self.h = h

    def tables(self):
        n = self.width * self.height
        pdf, cdf = np.zeros(n, np.float32), np.zeros(n, np.float32)
        ypdf, ycdf = np.zeros(self.height, np.float32), np.zeros(self.height, np.float32)
        tot = C.c_double()
        self.ctx.check(self.ctx.lib.dspbr_ibl_tables(self.h, fptr(pdf), fptr(cdf), fptr(ypdf), fptr(ycdf),
                                                     C.byref(tot)))
        return {"pdf": pdf, "cdf": cdf, "yPdf": ypdf, "yCdf": ycdf, "totalSum": tot.value}

    def alias_table(self):
        n = self.width * self.height
        prob, alias = np.zeros(n, np.float32), np.zeros(n, np.int32)
        self.ctx.check(self.ctx.lib.dspbr_ibl_alias_table(self.h, fptr(prob), iptr(alias)))
        return prob, alias

    def close(self):
        if self.h:
            self.ctx.lib.dspbr_ibl_destroy(self.h)
            self.h = None


@dataclass
class PathtracingCamera:
    """PathtracingCamera (renderer.ts:56-61): fov in degrees, near, matrixWorld."""
    matrixWorld: np.ndarray
    fov: float = 45.0
    near: float = 0.01


def look_at_matrix(position, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """ViewportCamera.setLookAt (pathtracing_viewport.ts:82-97)."""
    p, t, u = (np.asarray(x, np.float64) for x in (position, target, up))

    def nrm(v, fb):
        n = math.sqrt(float(v @ v))
        return np.asarray(fb, np.float64) if n <= 1e-10 else v / n

    fwd = nrm(t - p, (0, 0, -1))
    right = nrm(np.cross(fwd, u), (1, 0, 0))
    cam_up = nrm(np.cross(right, fwd), (0, 1, 0))
    e = np.zeros(16, np.float32)
    e[0:3], e[4:7], e[8:11], e[12:15], e[15] = right, cam_up, -fwd, p, 1.0
    return e


DISPLAY_SETTINGS = ("bvhBuilder", "wideBvh", "exposure", "toneMapping", "pixelRatio", "interactionPixelRatio", "enableGamma", "enableFxaa",
                    "tileResolution", "debugMode")


RESETTING_DISPLAY_SETTINGS = ("exposure", "enableGamma", "debugMode")


def render_resolution(display_w: int, display_h: int, pixel_ratio: float) -> tuple[int, int]:
    """renderRes = ceil(displayRes * pixelRatio) (renderer.ts:365-369), at least 1 x 1."""
    return max(1, math.ceil(display_w * pixel_ratio)), max(1, math.ceil(display_h * pixel_ratio))


def check_pixel_ratio(name: str, v) -> float:
    r = float(v)
    if not (r > 0.0 and math.isfinite(r)):
        raise ValueError(f"{name} must be a positive finite number, got {v!r}")
    return r


def apply_settings(p, settings: dict, display: dict | None = None) -> None:
    """PathtracingViewportSettings (pathtracing_viewport.ts:147-170) onto a
    dspbr_params; display-only keys go to `display` (or are ignored)."""
    for k, v in settings.items():
        if k == "maxBounces":
            p.max_bounces = int(v)
        elif k == "useIBL":
            p.use_ibl = int(bool(v))
        elif k == "showBackground":
            p.background_from_ibl = int(bool(v))
        elif k == "iblRotationDegrees":
            p.ibl_rotation_deg = float(v)
        elif k == "backgroundColor":
            for j in range(4):
                p.background_color[j] = float(v[j])
        elif k == "rayEps":
            p.ray_eps = float(v)
        elif k == "clampThreshold":
            p.clamp_threshold = float(v)
        elif k == "wideBvh":
            if v not in (4, 8):
                raise ValueError(f"wideBvh: {v!r} is not 4 or 8")
            if display is not None:
                display[k] = int(v)
        elif k in DISPLAY_SETTINGS:
            if display is not None:
                display[k] = v
        elif k == "rng":
            p.rng = _lib.RNG_PCG if v == "pcg" else _lib.RNG_MWC
        elif k == "seed":
            p.seed = int(v)
        elif k == "envSampling":
            p.env_sampling = _lib.ENV_CDF if v == "cdf" else _lib.ENV_ALIAS
        elif k == "russianRouletteStartDepth":
            p.rr_start_depth = int(v)
        elif k == "traversal":
            p.traversal = _lib.TRAVERSAL_REFERENCE if v == "reference" else _lib.TRAVERSAL_WIDE
        elif k == "bvhBuilder":
            if display is not None:
                display[k] = v

        elif k == "materialProfile":
            p.profile = _lib.PROFILE_LEAN if v == "webgl-lean" else _lib.PROFILE_FULL
        else:
            raise KeyError(f"unknown setting {k!r}")


class PathtracingViewport:
    """Drop-in for PathtracingViewport (pathtracing_viewport.ts:100-342) on a B200."""

    EVENTS = ("sceneLoaded", "sceneLoadFailed", "iblLoaded", "iblLoadFailed", "diagnosticsChanged",
              "frameRendered", "renderFinished")

    def __init__(self, settings: dict | None = None, device: int = 0, width: int = 1, height: int = 1,
                 materialProfile: str = "webgl-full"):
        self.ctx = Context(device)
        self.params = _lib.default_params()
        self.params.profile = _lib.PROFILE_LEAN if materialProfile == "webgl-lean" else _lib.PROFILE_FULL
        self._display = {"exposure": 1.0, "toneMapping": "None", "pixelRatio": 1.0, "interactionPixelRatio": 0.5,
                         "enableGamma": True, "enableFxaa": False, "tileResolution": 4, "debugMode": "None"}
        self._listeners: dict[str, set] = {e: set() for e in self.EVENTS}
        self._scene: DeviceScene | None = None
        self._ibl: DeviceIbl | None = None
        self.camera = PathtracingCamera(look_at_matrix((0, 0, 6), (0, 0, 0)), 45.0, 0.01)
        self.running = False
        self.interactionActive = False
        # displayWidth x displayHeight: the canvas (resize); width x height: the
        # render resolution the accumulation holds, scaled by the pixel ratio
        self.displayWidth, self.displayHeight = 0, 0
        self.width, self.height = 0, 0
        self._apply_params()
        self.resize(width, height)
        self._apply_camera()
        if settings:
            self.setSettings(settings)

    # ---- events (pathtracing_viewport.ts:125-143) ----
    def on(self, event: str, listener):
        self._listeners[event].add(listener)
        return lambda: self.off(event, listener)

    def off(self, event: str, listener):
        self._listeners[event].discard(listener)

    def _emit(self, event, payload):
        for fn in list(self._listeners[event]):
            fn(payload)

    # ---- settings (pathtracing_viewport.ts:147-170) ----
    def setSettings(self, settings: dict) -> None:
        for k in ("pixelRatio", "interactionPixelRatio"):
            if k in settings:
                check_pixel_ratio(k, settings[k])
        settings = dict(settings)
        if "pipelinedFrames" in settings:
            # not a reference setting: frames of consecutive accumulations
            # overlap on the device (dspbr_set_pipelining); start() then
            # returns once every sample has started, and readAccumulationAsync
            # of frames still in flight completes in readWait() or the next start().
            # True (or 2): two accumulations in flight; 3: three, for a caller
            # that takes each image two steps later (readWaitReady)
            self._set_pipelining(settings.pop("pipelinedFrames"))
        apply_settings(self.params, settings, self._display)
        # the renderer setters of exposure, enableGamma, debugMode and every
        # render setting reset the accumulation; toneMapping, enableFxaa,
        # and tileResolution do not (renderer.ts:172-306)
        if any(k not in DISPLAY_SETTINGS or k in RESETTING_DISPLAY_SETTINGS for k in settings):
            self._apply_params()
        # pixelRatio applies unless interaction mode is on, interactionPixelRatio
        # only while it is; the renderer's pixelRatio setter resizes, which
        # resets the accumulation (pathtracing_viewport.ts:150-157, renderer.ts:260-263)
        if ("pixelRatio" in settings and not self.interactionActive) or \
                ("interactionPixelRatio" in settings and self.interactionActive):
            self._apply_size()
        self._emit_diag()

    def setInteractionMode(self, active: bool) -> None:
        """pathtracing_viewport.ts:293-298: while the user interacts, render at
        interactionPixelRatio (0.5 by default) of the canvas resolution, else at
        pixelRatio; either way the accumulation restarts (renderer.ts:354-363)."""
        self.interactionActive = bool(active)
        self._apply_size()
        self._emit_diag()

    def _set_pipelining(self, v):
        depth = 2 if v is True else int(v)
        if v is not False and not 0 <= depth <= 16:
            raise ValueError(f"pipelinedFrames: {v!r} is not a bool or 2..16")
        on = v is not False and depth >= 2
        if on:
            self.ctx.check(self.ctx.lib.dspbr_set_pipeline_depth(self.ctx.h, depth))
        self.ctx.check(self.ctx.lib.dspbr_set_pipelining(self.ctx.h, int(on)))
        self._display["pipelinedFrames"] = depth if on else False

    def _pixel_ratio(self) -> float:
        return float(self._display["interactionPixelRatio" if self.interactionActive else "pixelRatio"])

    def _apply_size(self):
        """renderer.resize(displayRes): render resolution from the active pixel
        ratio; always resets the accumulation (renderer.ts:365-372)."""
        self.width, self.height = render_resolution(self.displayWidth, self.displayHeight, self._pixel_ratio())
        self._resize_device(self.width, self.height)

    def _resize_device(self, w: int, h: int):
        self.ctx.check(self.ctx.lib.dspbr_resize(self.ctx.h, w, h))

    def _apply_params(self):
        self.ctx.check(self.ctx.lib.dspbr_set_params(self.ctx.h, C.byref(self.params)))

    # ---- scene / IBL ----
    def setScene(self, scene) -> None:
        """scene: a synth.Scene or any object with vertices / indices / materials arrays."""
        try:
            self.ctx.set_bvh_builder(self._display.get("bvhBuilder", "device"))
            if "wideBvh" in self._display:
                self.ctx.set_wide_bvh(self._display["wideBvh"])
            ds = DeviceScene(self.ctx, scene.vertices, scene.indices, scene.materials, getattr(scene, "bvh", None))
            if getattr(scene, "tex_infos", None) is not None:
                ds.set_textures(scene.tex_infos, scene.tex_arrays)
        except Exception as e:
            self._emit("sceneLoadFailed", {"error": e})
            raise
        if self._scene is not None:
            self._scene.close()
        self._scene = ds
        ds.lights = list(getattr(scene, "lights", None) or [])
        if apply_scene_lights(self.params, ds.lights):
            self._apply_params()
        self.ctx.check(self.ctx.lib.dspbr_set_scene(self.ctx.h, ds.h))
        self._emit("sceneLoaded", {"scene": scene})
        self._emit_diag()

    def setIBL(self, ibl) -> None:
        """ibl: IblTextureLike ({'image': {'data', 'width', 'height'}}) or an (H, W, 4) array."""
        if isinstance(ibl, dict):
            im = ibl["image"]
            rgba = np.asarray(im["data"], np.float32).reshape(im["height"], im["width"], 4)
        else:
            rgba = np.asarray(ibl, np.float32)
        try:
            di = DeviceIbl(self.ctx, rgba)
        except Exception as e:
            self._emit("iblLoadFailed", {"error": e})
            raise
        if self._ibl is not None:
            self._ibl.close()
        self._ibl = di
        self.ctx.check(self.ctx.lib.dspbr_set_ibl(self.ctx.h, di.h))
        self._emit("iblLoaded", {"ibl": ibl})
        self._emit_diag()

    # ---- camera ----
    def setCamera(self, camera) -> None:
        self.camera = PathtracingCamera(f32(camera.matrixWorld).reshape(16), float(camera.fov), float(camera.near))
        self._apply_camera()
        self._emit_diag()

    def setLookAtCamera(self, position, target, up=(0.0, 1.0, 0.0), fov=None, near=None) -> None:
        self.camera = PathtracingCamera(look_at_matrix(position, target, up),
                                        self.camera.fov if fov is None else float(fov),
                                        self.camera.near if near is None else float(near))
        self._apply_camera()
        self._emit_diag()

    def _apply_camera(self):
        m = f32(self.camera.matrixWorld)
        self.ctx.check(self.ctx.lib.dspbr_set_camera(self.ctx.h, fptr(m), self.camera.fov, self.camera.near))

    # ---- size / progressive rendering ----
    def resize(self, width: int, height: int) -> None:
        """The canvas size (pathtracing_viewport.ts:255-260): max(1, floor(.))."""
        self.displayWidth, self.displayHeight = max(1, math.floor(width)), max(1, math.floor(height))
        self._apply_size()
        self._emit_diag()

    def start(self, sampleLimit: int = -1, frames_per_call: int | None = None) -> None:
        """Renders progressive frames until `sampleLimit` (synchronous; -1 = one frame)."""
        if self._scene is None:
            raise RuntimeError("Cannot start rendering without a scene.")
        self.running = True
        target = 1 if sampleLimit < 0 else int(sampleLimit)
        count = C.c_ulonglong(0)
        self.ctx.check(self.ctx.lib.dspbr_get_sample_count(self.ctx.h, C.byref(count)))
        done = int(count.value)
        while self.running and done < target:
            n = target - done if frames_per_call is None else min(frames_per_call, target - done)
            self.ctx.check(self.ctx.lib.dspbr_render(self.ctx.h, n))
            done += n
            self._emit("frameRendered", {"frameCount": done})
        self.running = False
        self._emit("renderFinished", {"frameCount": done})
        self._emit_diag()

    def stop(self) -> None:
        self.running = False
        self._emit_diag()

    def resetAccumulation(self) -> None:
        self.ctx.check(self.ctx.lib.dspbr_reset(self.ctx.h))
        self._emit_diag()

    def readAccumulation(self, out: np.ndarray | None = None) -> np.ndarray:
        """Running mean, (height, width, 4) float32 at the render resolution, row 0 = bottom row.

        With `out` (a C-contiguous float32 array of that shape, e.g. from
        allocReadbackBuffer()) the image is written there and `out` returned;
        otherwise a new array is returned."""
        shape = (self.height, self.width, 4)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"readAccumulation: out must be a C-contiguous float32 array of shape {shape}")
        self.ctx.check(self.ctx.lib.dspbr_read_accum(self.ctx.h, fptr(out), out.size))
        return out

    def readAccumulationAsync(self, out: np.ndarray) -> np.ndarray:
        """Pipelined readAccumulation into `out` (from allocReadbackBuffer():
        page-locked, (height, width, 4) float32): enqueues the mean and its
        copy and returns; the next start() overlaps the copy.  `out` holds
        the image after readWait()."""
        shape = (self.height, self.width, 4)
        if out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"readAccumulationAsync: out must be a C-contiguous float32 array of shape {shape}")
        self.ctx.check(self.ctx.lib.dspbr_read_accum_async(self.ctx.h, fptr(out), out.size))
        return out

    def readWait(self) -> None:
        """Waits for the copies of readAccumulationAsync."""
        self.ctx.check(self.ctx.lib.dspbr_read_wait(self.ctx.h))

    def readWaitReady(self) -> int:
        """Waits for the copies of readAccumulationAsync whose frames have
        finished and returns how many reads still wait for their frames
        (pipelined frames); renders nothing, unlike readWait()."""
        n = C.c_int()
        self.ctx.check(self.ctx.lib.dspbr_read_wait_ready(self.ctx.h, C.byref(n)))
        return n.value

    def readDisplay(self, rgba8: bool = True) -> np.ndarray:
        """The presented frame: the running mean through the reference's
        tone-mapping / gamma / FXAA passes with the viewport's display
        settings (exposure, toneMapping, enableGamma, enableFxaa;
        renderer.ts:666-700), drawn on the canvas (displayHeight, displayWidth,
        4): nearest-neighbour from the render resolution when the pixel ratio
        is not 1 (display.frag).  rgba8: the 8-bit canvas bytes, else RGBA32F."""
        d = _lib.display_params(canvas=(self.displayWidth, self.displayHeight), **self._display)
        shape = (self.displayHeight, self.displayWidth, 4)
        if rgba8:
            out = np.empty(shape, np.uint8)
            self.ctx.check(self.ctx.lib.dspbr_read_display_rgba8(self.ctx.h, C.byref(d),
                                                                 out.ctypes.data_as(C.POINTER(C.c_uint8)), out.size))
        else:
            out = np.empty(shape, np.float32)
            self.ctx.check(self.ctx.lib.dspbr_read_display(self.ctx.h, C.byref(d), fptr(out), out.size))
        return out

    def allocReadbackBuffer(self) -> np.ndarray:
        """A (height, width, 4) float32 array in page-locked host memory: the
        readback into it is a single device-to-host DMA.  Freed when the array
        is garbage collected."""
        return self.ctx.host_array((self.height, self.width, 4))

    @property
    def diagnostics(self) -> dict:
        d = _lib.Diag()
        self.ctx.check(self.ctx.lib.dspbr_get_diagnostics(self.ctx.h, C.byref(d)))
        out = d.as_dict()
        out["display"] = dict(self._display)
        out.update(self._resolution_diag())
        return out

    def _resolution_diag(self) -> dict:
        """renderResolution / displayResolution / mode as renderer.ts:971-976 reports them."""
        mode = "interactive" if self.interactionActive else ("accumulating" if self.running else "stopped")
        return {"renderResolution": f"{self.width}x{self.height}",
                "displayResolution": f"{self.displayWidth}x{self.displayHeight}", "mode": mode}

    def timeline(self, max_entries: int = 1024) -> np.ndarray:
        """(n, 3) float64: iteration, device clock (ms), paths queued after it;
        the last iterations of the path engine, oldest first."""
        n = max(1, min(int(max_entries), 1024))
        it, t, live = np.zeros(n, np.uint64), np.zeros(n, np.uint64), np.zeros(n, np.uint32)
        cnt = C.c_uint32()
        self.ctx.check(self.ctx.lib.dspbr_get_timeline(
            self.ctx.h, n, it.ctypes.data_as(C.POINTER(C.c_uint64)), t.ctypes.data_as(C.POINTER(C.c_uint64)),
            live.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(cnt)))
        k = cnt.value
        return np.stack([it[:k].astype(np.float64), t[:k].astype(np.float64) * 1e-6, live[:k].astype(np.float64)], 1)

    def _emit_diag(self):
        if self._listeners["diagnosticsChanged"]:
            self._emit("diagnosticsChanged", {"diagnostics": self.diagnostics})

    def dispose(self) -> None:
        self.stop()
        for o in (self._scene, self._ibl):
            if o is not None:
                o.close()
        self._scene = self._ibl = None
        self.ctx.close()
        for s in self._listeners.values():
            s.clear()


def createPathtracingViewport(**kw) -> PathtracingViewport:
    return PathtracingViewport(**kw)
