"""Host-side logic without a GPU: viewport settings semantics, display-mode
mapping, seeded request mixes, and the benchmark's multi-rank (replica)
reductions over gloo with world size 2."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

from dspbr import _lib, synth, viewport

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class _Recorder(viewport.PathtracingViewport):
    """PathtracingViewport whose device calls are recorded instead of made."""

    def __init__(self):
        self.params = _lib.default_params()
        self._display = {"exposure": 1.0, "toneMapping": "None", "enableGamma": True, "enableFxaa": False,
                         "pixelRatio": 1.0, "interactionPixelRatio": 0.5}
        self._listeners = {e: set() for e in self.EVENTS}
        self.applied = 0
        self.resizes = []  # render sizes given to dspbr_resize (each resets the accumulation)
        self.running = False
        self.interactionActive = False
        self.displayWidth = self.displayHeight = self.width = self.height = 0

    def _apply_params(self):
        self.applied += 1

    def _resize_device(self, w, h):
        self.resizes.append((w, h))

    @property
    def diagnostics(self):
        return self._resolution_diag()


def test_settings_reset_accumulation_like_the_reference_setters():
    v = _Recorder()
    # renderer.ts: tonemapping / enableFxaa setters keep the accumulation
    v.setSettings({"toneMapping": "AcesFilm"})
    v.setSettings({"enableFxaa": True, "tileResolution": 2, "interactionPixelRatio": 0.5})
    assert v.applied == 0
    # exposure / enableGamma / render settings reset it (renderer.ts:176-303)
    for s in ({"exposure": 2.0}, {"enableGamma": False}, {"maxBounces": 3}, {"rayEps": 1e-3},
              {"backgroundColor": [0, 0, 0, 1]}):
        before = v.applied
        v.setSettings(s)
        assert v.applied == before + 1, s
    assert v.params.max_bounces == 3 and abs(v.params.ray_eps - 1e-3) < 1e-9
    with pytest.raises(KeyError):
        v.setSettings({"noSuchSetting": 1})


def test_pixel_ratio_and_interaction_mode_set_the_render_resolution():
    # pathtracing_viewport.ts:147-160, 255-260, 293-298; renderer.ts:256-263, 354-372
    v = _Recorder()
    v.resize(801.7, 451)
    assert (v.displayWidth, v.displayHeight) == (801, 451) and v.resizes == [(801, 451)]
    assert v.diagnostics["renderResolution"] == "801x451" and v.diagnostics["mode"] == "stopped"
    # interaction mode: interactionPixelRatio (0.5) -> ceil(801 * 0.5) = 401, ceil(225.5) = 226
    v.setInteractionMode(True)
    assert v.resizes[-1] == (401, 226) and (v.width, v.height) == (401, 226)
    assert v.diagnostics == {"renderResolution": "401x226", "displayResolution": "801x451", "mode": "interactive"}
    # pixelRatio changes are stored but not applied while interacting ...
    n = len(v.resizes)
    v.setSettings({"pixelRatio": 2.0})
    assert len(v.resizes) == n
    # ... interactionPixelRatio applies at once (and resets)
    v.setSettings({"interactionPixelRatio": 0.25})
    assert v.resizes[-1] == (201, 113)
    # leaving interaction mode restores pixelRatio and resets even if the size is unchanged
    v.setInteractionMode(False)
    assert v.resizes[-1] == (1602, 902)
    v.setInteractionMode(False)
    assert v.resizes[-2:] == [(1602, 902), (1602, 902)]
    # outside interaction mode: pixelRatio applies, interactionPixelRatio is stored
    v.setSettings({"pixelRatio": 0.75})
    assert v.resizes[-1] == (601, 339)
    n = len(v.resizes)
    v.setSettings({"interactionPixelRatio": 0.5})
    assert len(v.resizes) == n and v._display["interactionPixelRatio"] == 0.5
    # a canvas resize keeps the ratio
    v.resize(100, 10)
    assert v.resizes[-1] == (75, 8)
    assert viewport.render_resolution(3, 3, 1e-9) == (1, 1)
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            v.setSettings({"pixelRatio": bad})
    # the canvas size reaches dspbr_display
    d = _lib.display_params(canvas=(801, 451))
    assert (d.canvas_width, d.canvas_height) == (801, 451)
    assert _lib.display_params().canvas_width == 0


def test_display_mode_mapping():
    # renderer.ts:192 tonemappingModes; indexOf() of an unknown name is -1
    assert _lib.display_params(toneMapping="None").tonemapping == 0
    assert _lib.display_params(toneMapping="AcesFilm").tonemapping == 3
    assert _lib.display_params(toneMapping="Uncharted2").tonemapping == -1
    d = _lib.display_params(exposure=2.5, enableGamma=False, enableFxaa=True)
    assert (d.exposure, d.gamma, d.fxaa) == (2.5, 0, 1)


def test_request_mix_is_seeded_and_in_range():
    a = synth.request_mix(3, 50, 8, 128 * 128, 1024 * 1024, 1, 64)
    b = synth.request_mix(3, 50, 8, 128 * 128, 1024 * 1024, 1, 64)
    assert [(r["scene"], r["width"], r["height"], r["spp"]) for r in a] == \
           [(r["scene"], r["width"], r["height"], r["spp"]) for r in b]
    for r in a:
        npx = r["width"] * r["height"]
        assert 0.9 * 128 * 128 <= npx <= 1.1 * 1024 * 1024
        assert 1 <= r["spp"] <= 64 and 0 <= r["scene"] < 8 and 30 <= r["camera"].fov <= 90


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": "2", "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench
    r, ws, local, dist = bench.dist_setup()
    mx = bench.reduce_max(dist, 1.5 + r)
    sm = bench.reduce_sum(dist, 1.0 + r)
    bench.barrier(dist)
    dist.destroy_process_group()
    q.put((r, ws, local, mx, sm))


def test_bench_replica_reductions_gloo_world_size_2():
    """bench.py --gpus N: every rank renders its own replica; device time is
    the max over ranks and rays the sum (no collective on the data path)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(k, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert [r[:3] for r in res] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == 2.5 and r[4] == 3.0 for r in res)


def test_first_scene_light_sets_the_point_light():
    # renderer.ts:424-430: lights[0] of any type, w = 1; no light: w = 0
    p = _lib.default_params()
    assert viewport.apply_scene_lights(p, [{"position": (1, 2, 3), "type": 1, "emission": (4, 5, 6)},
                                           {"position": (9, 9, 9), "type": 0, "emission": (1, 1, 1)}])
    assert tuple(p.point_light_position) == (1, 2, 3, 1) and tuple(p.point_light_emission) == (4, 5, 6, 1)
    assert not viewport.apply_scene_lights(p, [{"position": (1, 2, 3), "type": 0, "emission": (4, 5, 6)}])
    assert viewport.apply_scene_lights(p, [])
    assert tuple(p.point_light_position) == (0, 0, 0, 0)


def test_autotune_cache_round_trip(tmp_path):
    from dspbr import server
    path = str(tmp_path / "autotune.json")
    assert server.load_tuning(path) == {}
    a = {"path_pool": 1 << 22, "extend_blocks": 1184, "connect_blocks": 1036, "shade_blocks": 740}
    server.store_tuning(path, "NVIDIA B200|sm148|cc100|lib1-2", a)
    server.store_tuning(path, "other|sm1|cc00|lib3-4", dict(a, path_pool=1 << 20))
    d = server.load_tuning(path)
    assert d["NVIDIA B200|sm148|cc100|lib1-2"] == a and d["other|sm1|cc00|lib3-4"]["path_pool"] == 1 << 20
    with open(path, "w") as f:
        f.write("not json")
    assert server.load_tuning(path) == {}
    assert server.autotune_cache_path().endswith(os.path.join("dspbr", "autotune.json"))


def test_reference_arm_loads_no_library_of_this_repository():
    """bench.py --impl reference times the reference's shader compiled for the
    host (oracle/_ref); the workload's BVH is built by a child process, so the
    timing process maps no shared object of the product."""
    import subprocess
    code = ("import sys; sys.path.insert(0, %r); import bench; sc = bench.reference_workload(); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_LIB' if 'libdspbr_cuda' in maps else 'CLEAN', sc.bvh.nodes.size // 16, sc.num_triangles)"
            % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    word, nodes, tris = out.stdout.split()[-3:]
    assert word == "CLEAN" and int(nodes) > 0 and int(tris) > 1_000_000
