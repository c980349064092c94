"""Render server: continuous batching of viewport requests (dspbr_server_*).

Requests name a resident scene (DeviceScene) and IBL (DeviceIbl) of the
server's Context, a camera, a resolution, a sample count and viewport
settings.  The server admits them while path-pool slots and its HBM budget
allow, renders all admitted requests in the same launches, and writes each
mean image into the request's output array.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import _lib
from ._lib import check, f32
from .viewport import Context, DeviceIbl, DeviceScene, PathtracingCamera, apply_scene_lights, apply_settings

STATES = {_lib.REQ_QUEUED: "queued", _lib.REQ_RUNNING: "running", _lib.REQ_DONE: "done",
          _lib.REQ_CANCELLED: "cancelled", _lib.REQ_FAILED: "failed"}


def autotune_cache_path() -> str:
    """The autotuner's cache beside the shared library."""
    return os.path.join(os.path.dirname(os.path.abspath(_lib.LIB_PATH)), "autotune.json")


def load_tuning(path: str) -> dict:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def store_tuning(path: str, key: str, launch: dict) -> None:
    """Adds (or replaces) one GPU's entry; written to a temporary file and renamed."""
    d = load_tuning(path)
    d[key] = {k: int(v) for k, v in launch.items()}
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


class Server:
    def __init__(self, ctx: Context, path_pool: int = 0, max_active: int = 0, hbm_budget_bytes: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = _lib.ServerConfig()
        cfg.path_pool, cfg.max_active, cfg.hbm_budget_bytes = int(path_pool), int(max_active), int(hbm_budget_bytes)
        h = C.c_void_p()
        self.ctx.check(self.lib.dspbr_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self._out: dict[int, np.ndarray] = {}

    def close(self):
        if self.h:
            self.lib.dspbr_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        check(rc, self.ctx.h)

    def request(self, scene: DeviceScene, ibl: DeviceIbl | None, camera: PathtracingCamera, width: int, height: int,
                spp: int, settings: dict | None = None, out: np.ndarray | None = None, tag: int = 0):
        """Builds a dspbr_request (and its output array)."""
        r = _lib.Request()
        r.scene = scene.h.value if hasattr(scene.h, "value") else scene.h
        r.ibl = (ibl.h.value if hasattr(ibl.h, "value") else ibl.h) if ibl is not None else None
        m = f32(camera.matrixWorld).reshape(16)
        for i in range(16):
            r.camera[i] = float(m[i])
        r.fov_deg, r.near_plane = float(camera.fov), float(camera.near)
        r.width, r.height, r.spp = int(width), int(height), int(spp)
        self.lib.dspbr_params_default(C.byref(r.params))
        apply_scene_lights(r.params, getattr(scene, "lights", None))
        if settings:
            apply_settings(r.params, settings)
        if out is None:
            out = np.zeros((int(height), int(width), 4), np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size == width * height * 4
        r.out_rgba = out.ctypes.data_as(C.POINTER(C.c_float))
        r.tag = int(tag)
        return r, out

    def submit(self, *args, **kw) -> int:
        r, out = self.request(*args, **kw)
        rid = C.c_uint64()
        self._check(self.lib.dspbr_server_submit(self.h, C.byref(r), C.byref(rid)))
        self._out[rid.value] = out
        return rid.value

    def poll(self, rid: int) -> dict:
        info = _lib.RequestInfo()
        self._check(self.lib.dspbr_server_poll(self.h, rid, C.byref(info)))
        d = info.as_dict()
        d["state"] = STATES[d["state"]]
        return d

    def wait(self, rid: int, timeout_ms: int = -1) -> tuple[np.ndarray, dict]:
        """Blocks until the request finishes; returns (image, info)."""
        info = _lib.RequestInfo()
        self._check(self.lib.dspbr_server_wait(self.h, rid, int(timeout_ms), C.byref(info)))
        d = info.as_dict()
        d["state"] = STATES[d["state"]]
        return self._out[rid], d

    def cancel(self, rid: int) -> None:
        self._check(self.lib.dspbr_server_cancel(self.h, rid))

    def release(self, rid: int) -> None:
        self._check(self.lib.dspbr_server_release(self.h, rid))
        self._out.pop(rid, None)

    def stats(self) -> dict:
        st = _lib.ServerStats()
        self._check(self.lib.dspbr_server_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def autotune(self, samples: list, seconds: float = 10.0, cache: str | None = None) -> dict:
        """samples: requests from request(); renders them under candidate pool
        and block sizes and keeps the fastest.  Before the first submit.

        cache: a JSON file of earlier choices keyed by GPU (name, SM count,
        compute capability) and library build (size and modification time of
        the shared object), e.g. autotune_cache_path(): an entry for this GPU
        and build is applied without tuning; otherwise the tuner runs and its
        choice is added to the file.  Returns the stats with the launch sizes
        in use and "autotune_source" ("cache" or "tuned")."""
        key = self.tuning_key()
        if cache is not None:
            entry = load_tuning(cache).get(key)
            if entry is not None:
                self.set_launch(entry)
                return dict(self.stats(), autotune_source="cache")
        arr = (_lib.Request * len(samples))(*[s[0] if isinstance(s, tuple) else s for s in samples])
        self._check(self.lib.dspbr_server_autotune(self.h, arr, len(samples), float(seconds)))
        if cache is not None:
            store_tuning(cache, key, self.launch())
        return dict(self.stats(), autotune_source="tuned")

    def launch(self) -> dict:
        """Path pool and the grids of the persistent extend / connect / shade kernels in use."""
        lc = _lib.Launch()
        self._check(self.lib.dspbr_server_get_launch(self.h, C.byref(lc)))
        return lc.as_dict()

    def set_launch(self, launch: dict) -> None:
        lc = _lib.Launch()
        for k in ("path_pool", "extend_blocks", "connect_blocks", "shade_blocks"):
            setattr(lc, k, int(launch[k]))
        self._check(self.lib.dspbr_server_set_launch(self.h, C.byref(lc)))

    def tuning_key(self) -> str:
        info = _lib.DeviceInfo()
        self.ctx.check(self.lib.dspbr_get_device_info(self.ctx.h, C.byref(info)))
        st = os.stat(_lib.LIB_PATH)
        return (f"{info.name.decode()}|sm{info.sm_count}|cc{info.cc_major}{info.cc_minor}|"
                f"lib{st.st_size}-{int(st.st_mtime)}")
