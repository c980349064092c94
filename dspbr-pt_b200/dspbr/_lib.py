"""ctypes binding of libdspbr_cuda.so (include/dspbr.h).

The library is the product: every call goes to the CUDA implementation.  If
the shared object is missing the import fails loudly; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DSPBR_LIB", os.path.join(HERE, "libdspbr_cuda.so"))

OK = 0
ERR = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "invalid state",
       -5: "admission refused", -6: "not found", -7: "device fault"}
PROFILE_FULL, PROFILE_LEAN = 0, 1
RNG_MWC, RNG_PCG = 0, 1
ENV_ALIAS, ENV_CDF = 0, 1
TRAVERSAL_WIDE, TRAVERSAL_REFERENCE = 0, 1
BVH_BUILD_HOST, BVH_BUILD_DEVICE, BVH_BUILD_DEVICE_LBVH = 0, 1, 2


class DspbrError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERR.get(code, code)}: {message}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("max_bounces", C.c_int32), ("use_ibl", C.c_int32), ("ibl_rotation_deg", C.c_float),
        ("background_from_ibl", C.c_int32), ("background_color", C.c_float * 4), ("ray_eps", C.c_float),
        ("clamp_threshold", C.c_float), ("point_light_position", C.c_float * 4),
        ("point_light_emission", C.c_float * 4), ("rr_start_depth", C.c_int32), ("rr_termination_prob", C.c_float),
        ("profile", C.c_int32), ("rng", C.c_int32), ("seed", C.c_uint64), ("env_sampling", C.c_int32),
        ("traversal", C.c_int32), ("reserved", C.c_int32 * 6),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("sample_count", C.c_uint64), ("width", C.c_int32), ("height", C.c_int32),
        ("rays_primary", C.c_uint64), ("rays_extension", C.c_uint64), ("rays_shadow", C.c_uint64),
        ("traversal_aborted", C.c_uint64), ("scene_triangles", C.c_uint64), ("bvh_nodes", C.c_uint64),
        ("bvh_indices", C.c_uint64), ("device_bytes", C.c_uint64), ("last_render_ms", C.c_double),
        ("bvh_build_ms", C.c_double), ("upload_ms", C.c_double),
        ("nodes_closest", C.c_uint64), ("tris_closest", C.c_uint64), ("nodes_shadow", C.c_uint64),
        ("tris_shadow", C.c_uint64), ("extend_ms", C.c_double), ("connect_ms", C.c_double), ("shade_ms", C.c_double),
        ("extend_launches", C.c_uint64), ("connect_launches", C.c_uint64), ("shade_launches", C.c_uint64),
        ("other_launches", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TextureArray(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("layers", C.c_int32), ("rgba8", C.c_void_p)]


class Display(C.Structure):
    _fields_ = [("exposure", C.c_float), ("tonemapping", C.c_int32), ("gamma", C.c_int32), ("fxaa", C.c_int32),
                ("canvas_width", C.c_int32), ("canvas_height", C.c_int32), ("reserved", C.c_int32 * 2)]


TONEMAPPING_MODES = ["None", "Reinhard", "Cineon", "AcesFilm"]  # renderer.ts:192


def display_params(exposure=1.0, toneMapping="None", enableGamma=True, enableFxaa=False, canvas=None,
                   **_) -> Display:
    """Display settings of the viewport -> dspbr_display.  A mode name outside
    tonemappingModes selects no operator, as the reference's indexOf() = -1 does.
    canvas: (width, height) of the presented canvas, or None for the render size."""
    d = Display()
    d.exposure = float(exposure)
    d.tonemapping = TONEMAPPING_MODES.index(toneMapping) if toneMapping in TONEMAPPING_MODES else -1
    d.gamma = int(bool(enableGamma))
    d.fxaa = int(bool(enableFxaa))
    if canvas is not None:
        d.canvas_width, d.canvas_height = int(canvas[0]), int(canvas[1])
    return d


class ServerConfig(C.Structure):
    _fields_ = [("path_pool", C.c_uint32), ("max_active", C.c_int32), ("hbm_budget_bytes", C.c_uint64),
                ("reserved", C.c_int32 * 8)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("ibl", C.c_void_p), ("camera", C.c_float * 16), ("fov_deg", C.c_float),
                ("near_plane", C.c_float), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("params", Params), ("out_rgba", C.POINTER(C.c_float)), ("tag", C.c_uint64)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("tag", C.c_uint64), ("submit_ms", C.c_double), ("admit_ms", C.c_double),
                ("done_ms", C.c_double), ("device_bytes", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("cancelled", C.c_uint64), ("failed", C.c_uint64), ("queued", C.c_uint64), ("running", C.c_uint64),
                ("iterations", C.c_uint64), ("rays_closest", C.c_uint64), ("rays_shadow", C.c_uint64),
                ("bytes_in_use", C.c_uint64), ("bytes_peak", C.c_uint64), ("p50_ms", C.c_double),
                ("p99_ms", C.c_double), ("path_pool", C.c_uint32), ("trace_threads", C.c_int32),
                ("trace_blocks", C.c_int32), ("shade_threads", C.c_int32), ("shade_blocks", C.c_int32),
                ("connect_blocks", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Launch(C.Structure):
    _fields_ = [("path_pool", C.c_uint32), ("extend_blocks", C.c_int32), ("connect_blocks", C.c_int32),
                ("shade_blocks", C.c_int32), ("reserved", C.c_int32 * 4)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("sm_count", C.c_int32), ("cc_major", C.c_int32),
                ("cc_minor", C.c_int32), ("total_bytes", C.c_uint64)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED, REQ_FAILED = 0, 1, 2, 3, 4

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_U = C.POINTER(C.c_uint32)
_D = C.POINTER(C.c_double)
_V = C.c_void_p
_PV = C.POINTER(C.c_void_p)

SIGNATURES = {
    "dspbr_params_default": (None, [C.POINTER(Params)]),
    "dspbr_create": (C.c_int, [C.c_int, _PV]),
    "dspbr_destroy": (C.c_int, [_V]),
    "dspbr_last_error": (C.c_int, [_V, C.c_char_p, C.c_size_t]),
    "dspbr_device_count": (C.c_int, [_I]),
    "dspbr_bvh_build": (C.c_int, [_F, C.c_uint32, C.c_uint32, _U, C.c_uint32, _PV]),
    "dspbr_bvh_info": (C.c_int, [_V, _U, _U, _U, _U]),
    "dspbr_bvh_copy": (C.c_int, [_V, _F, _I]),
    "dspbr_bvh_error": (C.c_int, [_V, C.c_char_p, C.c_size_t]),
    "dspbr_bvh_free": (None, [_V]),
    "dspbr_bvh_wide": (C.c_int, [_F, C.c_uint32, C.c_uint32, _U, _U, _I, _F, _I]),
    "dspbr_scene_create": (C.c_int, [_V, _F, C.c_uint32, _U, C.c_uint32, _F, C.c_uint32, _F, C.c_uint32, _I,
                                      C.c_uint32, _PV]),
    "dspbr_set_bvh_builder": (C.c_int, [_V, C.c_int]),
    "dspbr_set_wide_bvh": (C.c_int, [_V, C.c_int]),
    "dspbr_scene_wide_bvh": (C.c_int, [_V, C.POINTER(C.c_int), _U, _U]),
    "dspbr_scene_set_textures": (C.c_int, [_V, _F, C.c_uint32, C.POINTER(TextureArray), C.c_uint32]),
    "dspbr_scene_bvh": (C.c_int, [_V, _F, _I, _U, _U]),
    "dspbr_scene_update_materials": (C.c_int, [_V, _F, C.c_uint32, C.c_uint32]),
    "dspbr_scene_update_vertices": (C.c_int, [_V, _F, C.c_uint32, C.c_uint32]),
    "dspbr_scene_device_bytes": (C.c_int, [_V, C.POINTER(C.c_uint64)]),
    "dspbr_scene_destroy": (C.c_int, [_V]),
    "dspbr_ibl_create": (C.c_int, [_V, _F, C.c_int, C.c_int, _PV]),
    "dspbr_ibl_tables": (C.c_int, [_V, _F, _F, _F, _F, _D]),
    "dspbr_ibl_alias_table": (C.c_int, [_V, _F, _I]),
    "dspbr_ibl_destroy": (C.c_int, [_V]),
    "dspbr_ibl_tables_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]),
    "dspbr_set_scene": (C.c_int, [_V, _V]),
    "dspbr_set_ibl": (C.c_int, [_V, _V]),
    "dspbr_set_camera": (C.c_int, [_V, _F, C.c_float, C.c_float]),
    "dspbr_set_params": (C.c_int, [_V, C.POINTER(Params)]),
    "dspbr_get_params": (C.c_int, [_V, C.POINTER(Params)]),
    "dspbr_resize": (C.c_int, [_V, C.c_int, C.c_int]),
    "dspbr_reset": (C.c_int, [_V]),
    "dspbr_render": (C.c_int, [_V, C.c_int]),
    "dspbr_render_async": (C.c_int, [_V, C.c_int]),
    "dspbr_poll": (C.c_int, [_V, _I]),
    "dspbr_wait": (C.c_int, [_V]),
    "dspbr_read_accum": (C.c_int, [_V, _F, C.c_size_t]),
    "dspbr_read_accum_async": (C.c_int, [_V, _F, C.c_size_t]),
    "dspbr_read_wait": (C.c_int, [_V]),
    "dspbr_set_pipelining": (C.c_int, [_V, C.c_int]),
    "dspbr_set_pipeline_depth": (C.c_int, [_V, C.c_int]),
    "dspbr_read_wait_ready": (C.c_int, [_V, C.POINTER(C.c_int)]),
    "dspbr_host_alloc": (C.c_int, [_V, C.c_size_t, C.POINTER(C.c_void_p)]),
    "dspbr_read_display": (C.c_int, [_V, C.POINTER(Display), _F, C.c_size_t]),
    "dspbr_read_display_rgba8": (C.c_int, [_V, C.POINTER(Display), C.POINTER(C.c_uint8), C.c_size_t]),
    "dspbr_display_image": (C.c_int, [_V, _F, C.c_int, C.c_int, C.POINTER(Display), _F, C.POINTER(C.c_uint8)]),
    "dspbr_host_free": (C.c_int, [_V, _V]),
    "dspbr_get_diagnostics": (C.c_int, [_V, C.POINTER(Diag)]),
    "dspbr_get_sample_count": (C.c_int, [_V, C.POINTER(C.c_ulonglong)]),
    "dspbr_get_timeline": (C.c_int, [_V, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "dspbr_set_wave_paths": (C.c_int, [_V, C.c_uint32]),
    "dspbr_set_drain_threshold": (C.c_int, [_V, C.c_uint32]),
    "dspbr_set_counting": (C.c_int, [_V, C.c_int]),
    "dspbr_set_profiling": (C.c_int, [_V, C.c_int]),
    "dspbr_trace_closest": (C.c_int, [_V, _V, _F, C.c_uint32, _I, _F, _F]),
    "dspbr_trace_occluded": (C.c_int, [_V, _V, _F, C.c_uint32, _I]),
    "dspbr_bsdf_query": (C.c_int, [_V, _V, C.c_uint32, _F, _F, _F, _F, _F, _I]),
    "dspbr_ibl_query": (C.c_int, [_V, _V, C.c_uint32, _F, _F, _F, _F, _F]),
    "dspbr_camera_rays": (C.c_int, [_V, C.c_uint32, _I, _F, _F]),
    "dspbr_server_create": (C.c_int, [_V, C.POINTER(ServerConfig), _PV]),
    "dspbr_server_submit": (C.c_int, [_V, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "dspbr_server_poll": (C.c_int, [_V, C.c_uint64, C.POINTER(RequestInfo)]),
    "dspbr_server_wait": (C.c_int, [_V, C.c_uint64, C.c_int, C.POINTER(RequestInfo)]),
    "dspbr_server_cancel": (C.c_int, [_V, C.c_uint64]),
    "dspbr_server_release": (C.c_int, [_V, C.c_uint64]),
    "dspbr_server_get_stats": (C.c_int, [_V, C.POINTER(ServerStats)]),
    "dspbr_server_autotune": (C.c_int, [_V, C.POINTER(Request), C.c_int, C.c_double]),
    "dspbr_server_get_launch": (C.c_int, [_V, C.POINTER(Launch)]),
    "dspbr_server_set_launch": (C.c_int, [_V, C.POINTER(Launch)]),
    "dspbr_get_device_info": (C.c_int, [_V, C.POINTER(DeviceInfo)]),
    "dspbr_server_destroy": (C.c_int, [_V]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libdspbr_cuda.so not found at {path}: build it with dspbr-pt_b200/build.py")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_F)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def uptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def check(rc: int, ctx=None) -> None:
    if rc != OK:
        msg = ""
        if ctx is not None:
            buf = C.create_string_buffer(512)
            load().dspbr_last_error(ctx, buf, 512)
            msg = buf.value.decode(errors="replace")
        raise DspbrError(rc, msg)


def default_params() -> Params:
    p = Params()
    load().dspbr_params_default(C.byref(p))
    return p
