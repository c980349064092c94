"""Seeded synthetic scenes and environment maps in the reference's packed formats.

The reference has no bundled test assets (its glTF sample models and HDRIs are
fetched by URL at run time), so every workload here is generated:

* vertices: 20 float32 per vertex — position.xyz + material index, normal.xyz + 0,
  uv0.xy + uv1.xy, tangent.xyzw, colour.rgba (scene_loader.ts:296-344,
  VERTEX_STRIDE scene_data.ts:21).  Meshes without tangents carry zeros, as the
  loader leaves them, so the shader falls back to get_onb (bvh.glsl:129-134);
* indices: uint32, 3 per triangle;
* materials: 68 float32 per material, defaults of MaterialData's constructor
  (material.ts:436-480), field offsets of material.ts:25-413;
* environment maps: RGBA32F, row 0 = zenith (dir_to_uv, utils.glsl:141-147).

Workloads (sizes of the benchmark configurations):
  small       ~1.3k tris, 512x512, 64 spp, 8 bounces, env 256x128
  large       ~1M tris (256 instances), 1920x1080, 256 spp, 12 bounces, env 2048x1024
  divergence  ~4M tris, 60% transmissive/volume, 20% iridescent, 1280x720,
              512 spp, 32 bounces, Russian roulette after bounce 4, env 4096x2048
  sized(n)    scenes of a given triangle count for the batching/serving mixes
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

VERTEX_STRIDE = 20
MATERIAL_STRIDE = 68

# material.ts field offsets (setters at material.ts:25-413)
MAT = {
    "baseColorFactor": 0, "metallicFactor": 3, "roughnessFactor": 4, "anisotropy": 5,
    "anisotropyRotation": 6, "transmissionFactor": 7, "cutoutOpacity": 8, "doubleSided": 9,
    "normalScale": 10, "ior": 11, "specularColorFactor": 12, "specularFactor": 15,
    "sheenColorFactor": 16, "sheenRoughnessFactor": 19, "emissiveFactor": 20,
    "clearcoatNormalTextureScale": 23, "clearcoatFactor": 24, "clearcoatRoughnessFactor": 25,
    "diffuseTransmissionFactor": 26, "alphaCutoff": 27, "attenuationColor": 28,
    "attenuationDistance": 31, "multiscatterColorFactor": 32, "thinWalled": 35,
    "anisotropyDirection": 36, "diffuseTransmissionTextureId": 39, "iridescenceFactor": 40,
    "iridescenceIor": 41, "iridescenceThicknessMinimum": 42, "iridescenceThicknessMaximum": 43,
    "baseColorTextureId": 44, "metallicRoughnessTextureId": 45, "normalTextureId": 46,
    "emissiveTextureId": 47, "specularTextureId": 48, "specularColorTextureId": 49,
    "transmissionTextureId": 50, "clearcoatTextureId": 51, "clearcoatRoughnessTextureId": 52,
    "clearcoatNormalTextureId": 53, "sheenColorTextureId": 54, "sheenRoughnessTextureId": 55,
    "anisotropyTextureId": 56, "anisotropyDirectionTextureId": 57, "iridescenceTextureId": 58,
    "iridescenceThicknessTextureId": 59, "diffuseTransmissionColorFactor": 60,
    "diffuseTransmissionColorTextureId": 63, "dispersion": 64,
}


def default_material() -> np.ndarray:
    """MaterialData() defaults (material.ts:436-480)."""
    m = np.zeros(MATERIAL_STRIDE, np.float32)

    def put(name, v):
        o = MAT[name]
        v = np.atleast_1d(np.asarray(v, np.float64))
        m[o:o + v.size] = v

    put("baseColorFactor", [1, 1, 1]); put("metallicFactor", 0); put("roughnessFactor", 0)
    put("anisotropy", 0); put("anisotropyRotation", 0); put("transmissionFactor", 0)
    put("cutoutOpacity", 1); put("doubleSided", 1); put("normalScale", 1); put("ior", 1.49)
    put("specularColorFactor", [1, 1, 1]); put("specularFactor", 1)
    put("sheenRoughnessFactor", 0); put("sheenColorFactor", [0, 0, 0])
    put("clearcoatNormalTextureScale", 1); put("emissiveFactor", [0, 0, 0])
    put("clearcoatFactor", 0); put("clearcoatRoughnessFactor", 0)
    put("diffuseTransmissionFactor", 0); put("alphaCutoff", 0)
    m[MAT["attenuationDistance"]] = np.float32(np.inf)  # Number.MAX_VALUE -> Float32Array
    put("attenuationColor", [1, 1, 1]); put("multiscatterColorFactor", [1, 1, 1]); put("thinWalled", 1)
    put("anisotropyDirection", [1, 0, 0]); put("diffuseTransmissionTextureId", -1)
    put("iridescenceFactor", 0); put("iridescenceIor", 1.3)
    put("iridescenceThicknessMinimum", 100); put("iridescenceThicknessMaximum", 400)
    for k in MAT:
        if k.endswith("TextureId"):
            m[MAT[k]] = -1
    put("diffuseTransmissionColorFactor", [1, 1, 1]); put("dispersion", 0)
    return m


def set_field(m: np.ndarray, name: str, value) -> None:
    o = MAT[name]
    v = np.atleast_1d(np.asarray(value, np.float64)).astype(np.float32)
    m[o:o + v.size] = v


@dataclass
class Camera:
    matrix_world: np.ndarray  # 16 floats, column-major camera-to-world
    fov: float = 45.0
    near: float = 0.1

    @staticmethod
    def look_at(position, target, up=(0.0, 1.0, 0.0), fov=45.0, near=0.1) -> "Camera":
        """ViewportCamera.setLookAt (pathtracing_viewport.ts:82-97)."""
        p = np.asarray(position, np.float64)
        t = np.asarray(target, np.float64)
        u = np.asarray(up, np.float64)

        def nrm(v, fb):
            n = np.linalg.norm(v)
            return np.asarray(fb, np.float64) if n <= 1e-10 else v / n

        fwd = nrm(t - p, (0, 0, -1))
        right = nrm(np.cross(fwd, u), (1, 0, 0))
        cam_up = nrm(np.cross(right, fwd), (0, 1, 0))
        back = -fwd
        e = np.zeros(16, np.float32)
        e[0:3] = right; e[4:7] = cam_up; e[8:11] = back; e[12:15] = p; e[15] = 1
        return Camera(e, float(fov), float(near))


@dataclass
class Scene:
    name: str
    vertices: np.ndarray          # (V, 20) float32
    indices: np.ndarray           # (3T,) uint32
    materials: np.ndarray         # (M, 68) float32
    camera: Camera
    width: int = 512
    height: int = 512
    spp: int = 64
    max_bounces: int = 8
    rr_start_depth: int = 2
    env: np.ndarray | None = None  # (H, W, 4) float32
    seed: int = 0
    meta: dict = field(default_factory=dict)
    # KHR_lights_punctual lights on mesh nodes, as scene_loader.ts:187-199 adds
    # them: {"position": (x, y, z), "type": 0 point / 1 other, "emission": (r, g, b)}
    lights: list = field(default_factory=list)

    @property
    def num_triangles(self) -> int:
        return self.indices.size // 3

    def positions(self) -> np.ndarray:
        return np.ascontiguousarray(self.vertices[:, 0:3])


# ---- mesh primitives --------------------------------------------------------
def icosphere(level: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.asarray(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = f
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.asarray(verts, np.float64), np.asarray(faces, np.int64)


def grid(nx: int, ny: int):
    xs = np.linspace(-0.5, 0.5, nx + 1)
    ys = np.linspace(-0.5, 0.5, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="xy")
    verts = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], 1)
    uv = np.stack([(X.ravel() + 0.5), (Y.ravel() + 0.5)], 1)
    i = np.arange(ny)[:, None] * (nx + 1) + np.arange(nx)[None, :]
    a, b, c, d = i, i + 1, i + nx + 1, i + nx + 2
    faces = np.concatenate([np.stack([a, b, d], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    return verts, faces, uv


def vertex_normals(verts, faces):
    fn = np.cross(verts[faces[:, 1]] - verts[faces[:, 0]], verts[faces[:, 2]] - verts[faces[:, 0]])
    n = np.zeros_like(verts)
    for k in range(3):
        np.add.at(n, faces[:, k], fn)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return n / np.maximum(ln, 1e-20)


def random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


class MeshBuilder:
    def __init__(self):
        self.v: list[np.ndarray] = []
        self.f: list[np.ndarray] = []
        self.count = 0

    def add(self, pos, faces, normals, mat, uv=None, flat=False):
        pos = np.asarray(pos, np.float64)
        faces = np.asarray(faces, np.int64)
        if flat:  # unshared vertices with the face normal
            p = pos[faces.reshape(-1)]
            fn = np.cross(p[1::3] - p[0::3], p[2::3] - p[0::3])
            fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-20)
            normals = np.repeat(fn, 3, axis=0)
            uv = None if uv is None else np.asarray(uv)[faces.reshape(-1)]
            pos = p
            faces = np.arange(p.shape[0]).reshape(-1, 3)
        rec = np.zeros((pos.shape[0], VERTEX_STRIDE), np.float32)
        rec[:, 0:3] = pos
        rec[:, 3] = mat
        rec[:, 4:7] = normals
        if uv is not None:
            rec[:, 8:10] = uv
        rec[:, 16:20] = 1.0
        self.v.append(rec)
        self.f.append(faces + self.count)
        self.count += pos.shape[0]

    def arrays(self):
        return np.concatenate(self.v), np.concatenate(self.f).astype(np.uint32).reshape(-1)


# ---- environment maps -------------------------------------------------------
def _texel_dirs(w, h):
    """Direction of each texel centre, inverse of dir_to_uv (utils.glsl:141-154)."""
    u = (np.arange(w) + 0.5) / w
    v = (np.arange(h) + 0.5) / h
    phi = u[None, :] * 2 * np.pi
    theta = v[:, None] * np.pi
    return np.stack([np.sin(theta) * np.cos(phi), np.cos(theta) * np.ones_like(phi),
                     np.sin(theta) * np.sin(phi)], -1)


def env_sun(w, h, base, sun_dir, peak, sigma_deg):
    d = _texel_dirs(w, h)
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    ang = np.arccos(np.clip(d @ s, -1, 1))
    lum = base + peak * np.exp(-0.5 * (ang / np.radians(sigma_deg)) ** 2)
    env = np.ones((h, w, 4), np.float32)
    env[..., :3] = lum[..., None]
    return env


def env_lognormal(w, h, rng, sigma=1.5, sun_peak=1e4, sun_sigma_deg=1.0):
    lum = np.exp(rng.normal(0.0, sigma, size=(h, w)))
    tint = rng.uniform(0.7, 1.0, size=(h, w, 3))
    env = np.ones((h, w, 4), np.float32)
    env[..., :3] = lum[..., None] * tint
    sun = np.array([rng.uniform(-1, 1), rng.uniform(0.3, 1.0), rng.uniform(-1, 1)])
    d = _texel_dirs(w, h)
    ang = np.arccos(np.clip(d @ (sun / np.linalg.norm(sun)), -1, 1))
    env[..., :3] += (sun_peak * np.exp(-0.5 * (ang / np.radians(sun_sigma_deg)) ** 2))[..., None]
    return env


# ---- materials ---------------------------------------------------------------
def random_base_material(rng):
    m = default_material()
    set_field(m, "baseColorFactor", rng.uniform(0.1, 0.9, 3))
    set_field(m, "roughnessFactor", rng.uniform(0.05, 1.0))
    set_field(m, "metallicFactor", float(rng.integers(0, 2)))
    return m


def glass_material(ior=1.5):
    m = default_material()
    set_field(m, "baseColorFactor", [1, 1, 1])
    set_field(m, "roughnessFactor", 0.0)
    set_field(m, "transmissionFactor", 1.0)
    set_field(m, "ior", ior)
    set_field(m, "thinWalled", 0.0)
    return m


def feature_material(rng, kind: str):
    """One material per DSPBR feature class, parameters drawn as in the large config."""
    m = random_base_material(rng)
    if kind == "anisotropy":
        set_field(m, "metallicFactor", 1.0)
        set_field(m, "anisotropy", rng.uniform(-1, 1))
        rot = rng.uniform(0, 2 * np.pi)
        set_field(m, "anisotropyDirection", [math.cos(rot), math.sin(rot), 0.0])
    elif kind == "clearcoat":
        set_field(m, "clearcoatFactor", rng.uniform(0, 1))
        set_field(m, "clearcoatRoughnessFactor", rng.uniform(0, 1))
    elif kind == "sheen":
        set_field(m, "metallicFactor", 0.0)
        set_field(m, "sheenColorFactor", rng.uniform(0, 1, 3))
        set_field(m, "sheenRoughnessFactor", rng.uniform(0, 1))
    elif kind == "transmission":
        set_field(m, "metallicFactor", 0.0)
        set_field(m, "transmissionFactor", 1.0)
        set_field(m, "ior", rng.uniform(1.3, 1.8))
        set_field(m, "roughnessFactor", rng.uniform(0.0, 0.3))
        set_field(m, "thinWalled", float(rng.integers(0, 2)))
    elif kind == "volume":
        set_field(m, "metallicFactor", 0.0)
        set_field(m, "transmissionFactor", 1.0)
        set_field(m, "ior", rng.uniform(1.3, 1.8))
        set_field(m, "roughnessFactor", rng.uniform(0.0, 0.3))
        set_field(m, "thinWalled", 0.0)
        set_field(m, "attenuationDistance", 10 ** rng.uniform(-1, 1))
        set_field(m, "attenuationColor", rng.uniform(0.2, 1.0, 3))
    elif kind == "iridescence":
        set_field(m, "iridescenceFactor", 1.0)
        set_field(m, "iridescenceIor", rng.uniform(1.2, 2.0))
        set_field(m, "iridescenceThicknessMaximum", rng.uniform(100, 400))
    elif kind == "dispersion":
        set_field(m, "metallicFactor", 0.0)
        set_field(m, "transmissionFactor", 1.0)
        set_field(m, "ior", rng.uniform(1.3, 1.8))
        set_field(m, "roughnessFactor", rng.uniform(0.0, 0.2))
        set_field(m, "thinWalled", 0.0)
        set_field(m, "dispersion", 20.0 / rng.uniform(20, 60))  # KHR: 20 / Abbe number
        set_field(m, "attenuationColor", rng.uniform(0.2, 1.0, 3))
        set_field(m, "attenuationDistance", 10 ** rng.uniform(-1, 1))
    return m


FEATURES = ["base", "anisotropy", "clearcoat", "sheen", "transmission", "volume", "iridescence", "dispersion"]


# ---- workloads ---------------------------------------------------------------
def make_small(seed: int = 0) -> Scene:
    """Cornell-style box (10 quads) + two boxes + level-3 icosphere = 1,324 tris."""
    rng = np.random.default_rng(seed)
    mb = MeshBuilder()
    mats = [random_base_material(rng) for _ in range(7)] + [glass_material(1.5)]
    # five walls, each two quads (open towards +z)
    walls = [
        ((-1, 0, -1), (2, 0, 0), (0, 0, 2)),   # floor
        ((-1, 2, 1), (2, 0, 0), (0, 0, -2)),   # ceiling
        ((-1, 0, -1), (0, 2, 0), (2, 0, 0)),   # back
        ((-1, 0, 1), (0, 2, 0), (0, 0, -2)),   # left
        ((1, 0, -1), (0, 2, 0), (0, 0, 2)),    # right
    ]
    for wi, (o, a, b) in enumerate(walls):
        o, a, b = (np.asarray(x, np.float64) for x in (o, a, b))
        for half in range(2):
            oo = o + a * 0.5 * half
            p = np.stack([oo, oo + a * 0.5, oo + a * 0.5 + b, oo + b])
            mb.add(p, [[0, 1, 2], [0, 2, 3]], None, wi, uv=[[0, 0], [1, 0], [1, 1], [0, 1]], flat=True)
    # two boxes
    for bi, (c, s, ang) in enumerate([((-0.35, 0.6, -0.3), (0.55, 1.2, 0.55), 0.3),
                                      ((0.4, 0.3, 0.35), (0.55, 0.6, 0.55), -0.3)]):
        corners = np.array([[x, y, z] for x in (-.5, .5) for y in (-.5, .5) for z in (-.5, .5)]) * s
        R = np.array([[math.cos(ang), 0, math.sin(ang)], [0, 1, 0], [-math.sin(ang), 0, math.cos(ang)]])
        corners = corners @ R.T + np.asarray(c)
        faces = [[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                 [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]]
        mb.add(corners, faces, None, 5 + bi, flat=True)
    sv, sf = icosphere(3)
    mb.add(sv * 0.35 + np.array([0.35, 0.95, 0.35]), sf, sv, 7)
    verts, idx = mb.arrays()
    sun = [rng.uniform(-0.5, 0.5), rng.uniform(0.5, 1.0), rng.uniform(0.2, 1.0)]
    env = env_sun(256, 128, 0.3, sun, 500.0, 2.0)
    cam = Camera.look_at((0, 1, 3.6), (0, 1, 0), fov=45.0, near=0.1)
    return Scene("small", verts, idx, np.stack(mats), cam, 512, 512, 64, 8, 2, env, seed,
                 {"sun": sun})


def _instances(rng, n_inst, tris_per_inst, mat_kinds, cube=100.0, materials_out=None):
    """Seeded displaced grids and icospheres with random transforms in a cube."""
    mb = MeshBuilder()
    level = max(1, int(round(math.log(max(tris_per_inst, 20) / 20.0, 4))))
    sv, sf = icosphere(level)
    side = max(2, int(round(math.sqrt(tris_per_inst / 2.0))))
    gv, gf, guv = grid(side, side)
    mats = []
    for i in range(n_inst):
        kind = mat_kinds[i % len(mat_kinds)] if isinstance(mat_kinds, list) else mat_kinds(i)
        mats.append(feature_material(rng, kind))
        R = random_rotation(rng)
        s = rng.uniform(2.0, 8.0)
        t = rng.uniform(-cube / 2, cube / 2, 3)
        if i % 2 == 0:
            amp = rng.uniform(0.02, 0.15)
            fx, fy = rng.uniform(1, 6, 2)
            ph = rng.uniform(0, 2 * np.pi, 2)
            p = gv.copy()
            p[:, 2] = amp * np.sin(2 * np.pi * fx * p[:, 0] + ph[0]) * np.cos(2 * np.pi * fy * p[:, 1] + ph[1])
            n = vertex_normals(p, gf)
            mb.add((p * s) @ R.T + t, gf, n @ R.T, i, uv=guv)
        else:
            mb.add((sv * s * 0.5) @ R.T + t, sf, sv @ R.T, i)
    verts, idx = mb.arrays()
    return verts, idx, np.stack(mats)


def make_large(seed: int = 0, target_tris: int = 1_000_000, n_inst: int = 256) -> Scene:
    rng = np.random.default_rng(seed)
    verts, idx, mats = _instances(rng, n_inst, target_tris // n_inst, FEATURES)
    env = env_lognormal(2048, 1024, rng, 1.5, 1e4)
    cam = Camera.look_at((0, 15, 135), (0, 0, 0), fov=45.0, near=0.1)
    return Scene("large", verts, idx, mats, cam, 1920, 1080, 256, 12, 2, env, seed)


def make_large_framed(seed: int = 0) -> Scene:
    """The large configuration seen by a camera at the edge of the instance
    cloud's 100 m cube that frames the cloud: 72% of 1080p primary rays hit
    geometry (against 20% for make_large's camera outside the cube), so most
    paths bounce, shade and trace shadow rays."""
    sc = make_large(seed)
    sc.name = "large_framed"
    sc.camera = Camera.look_at((-48.0, 28.0, -33.0), (0.0, 5.0, -14.0), fov=46.0, near=0.1)
    return sc


def _divergence_kind(i):
    """60% transmissive / volume / dispersive, 20% iridescent, 20% base materials."""
    r = (i * 7919) % 10
    if r < 6:
        return ["transmission", "volume", "dispersion"][r % 3]
    return "iridescence" if r < 8 else "base"


def make_divergence(seed: int = 0, n_inst: int = 536, tris_per_inst: int = 10_000) -> Scene:
    """~4.0M triangles: 536 instances alternating 9,800-triangle displaced grids
    and 5,120-triangle icospheres."""
    rng = np.random.default_rng(seed)
    verts, idx, mats = _instances(rng, n_inst, tris_per_inst, _divergence_kind)
    env = env_lognormal(4096, 2048, rng, 1.5, 1e4)
    cam = Camera.look_at((0, 15, 135), (0, 0, 0), fov=45.0, near=0.1)
    return Scene("divergence", verts, idx, mats, cam, 1280, 720, 512, 32, 4, env, seed)


def make_divergence_small(seed: int = 0) -> Scene:
    """The divergence configuration's material mix on a small scene for
    path-level parity: 24 instances (~5.4k triangles) packed in a 12 m cube,
    128x64 environment, 32 bounces."""
    rng = np.random.default_rng(seed)
    verts, idx, mats = _instances(rng, 24, 320, _divergence_kind, cube=12.0)
    env = env_lognormal(128, 64, rng, 1.5, 1e3)
    cam = Camera.look_at((0, 4, 18), (0, 0, 0), fov=50.0, near=0.05)
    return Scene("divergence-small", verts, idx, mats, cam, 48, 36, 16, 32, 2, env, seed)


def make_sized(seed: int, target_tris: int, env_size=(1024, 512)) -> Scene:
    """Scene of about `target_tris` triangles for the batching / serving mixes."""
    rng = np.random.default_rng(seed)
    n_inst = int(np.clip(target_tris // 4000, 4, 256))
    verts, idx, mats = _instances(rng, n_inst, max(20, target_tris // n_inst), FEATURES)
    env = env_lognormal(env_size[0], env_size[1], rng, 1.5, 1e4)
    cam = Camera.look_at((0, 15, 135), (0, 0, 0), fov=45.0, near=0.1)
    return Scene(f"sized{target_tris}", verts, idx, mats, cam, 512, 512, 16, 12, 2, env, seed)


# ---- material textures --------------------------------------------------------
TEXTURE_SLOTS = ["baseColorTextureId", "metallicRoughnessTextureId", "normalTextureId", "emissiveTextureId",
                 "specularTextureId", "specularColorTextureId", "transmissionTextureId", "clearcoatTextureId",
                 "clearcoatRoughnessTextureId", "sheenColorTextureId", "sheenRoughnessTextureId",
                 "anisotropyTextureId", "anisotropyDirectionTextureId", "iridescenceTextureId",
                 "iridescenceThicknessTextureId", "diffuseTransmissionTextureId",
                 "diffuseTransmissionColorTextureId"]


def texture_set(seed: int = 0):
    """Seeded material textures as the reference packs them (scene_data.ts:71-100):
    RGBA8 arrays grouped by resolution, and TexInfo records (offset.xy, array,
    layer, scale.xy, uv set, pad; material.ts:483-523).  Array 0 is 32x32 with
    5 layers (colour checker with alpha, occlusion-roughness-metallic noise,
    normal-map bumps, emissive dots, masks); array 1 is 16x8 with 2 layers."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:32, 0:32]
    a0 = np.zeros((5, 32, 32, 4), np.uint8)
    chk = ((x // 8 + y // 8) % 2).astype(bool)
    a0[0, ..., 0] = np.where(chk, 220, 40)
    a0[0, ..., 1] = np.where(chk, 180, 90)
    a0[0, ..., 2] = rng.integers(30, 230, (32, 32))
    a0[0, ..., 3] = np.where((x + y) % 11 == 0, 60, 255)
    a0[1, ..., 0] = 255
    a0[1, ..., 1] = rng.integers(10, 255, (32, 32))
    a0[1, ..., 2] = rng.integers(0, 255, (32, 32))
    a0[1, ..., 3] = 255
    bump = np.sin(x / 32 * 2 * np.pi * 3)[..., None] * np.array([0.4, 0.0, 0.0]) + \
        np.cos(y / 32 * 2 * np.pi * 2)[..., None] * np.array([0.0, 0.3, 0.0])
    nrm = bump + np.array([0.0, 0.0, 1.0])
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    a0[2, ..., 0:3] = np.round((nrm * 0.5 + 0.5) * 255).astype(np.uint8)
    a0[2, ..., 3] = 255
    dots = ((x % 9 == 4) & (y % 7 == 3))
    a0[3, ..., 0:3] = np.where(dots[..., None], np.array([255, 200, 120]), 0)
    a0[3, ..., 3] = 255
    a0[4] = rng.integers(0, 256, (32, 32, 4))
    y1, x1 = np.mgrid[0:8, 0:16]
    a1 = np.zeros((2, 8, 16, 4), np.uint8)
    a1[0, ..., 0:3] = rng.integers(60, 256, (8, 16, 3))
    a1[0, ..., 3] = rng.integers(0, 256, (8, 16))
    ang = np.arctan2(y1 - 3.5, x1 - 7.5)
    a1[1, ..., 0] = np.round((np.cos(ang) * 0.5 + 0.5) * 255)
    a1[1, ..., 1] = np.round((np.sin(ang) * 0.5 + 0.5) * 255)
    a1[1, ..., 2] = rng.integers(0, 256, (8, 16))
    a1[1, ..., 3] = 255
    # (array, layer, scale, offset, uv set)
    refs = [(0, 0, (1, 1), (0, 0), 0), (0, 1, (2.5, 1.5), (0.3, -0.2), 0), (0, 2, (1, 1), (0, 0), 0),
            (0, 3, (3, 3), (0.1, 0.7), 0), (0, 4, (0.5, 2), (0.25, 0), 0), (1, 0, (1, 1), (0, 0), 0),
            (1, 1, (1.7, 0.9), (-0.4, 0.15), 0), (0, 0, (4, 4), (0.5, 0.5), 1), (1, 0, (6, 2), (0, 0), 0)]
    infos = np.zeros((len(refs), 8), np.float32)
    for k, (arr, layer, sc, off, uvset) in enumerate(refs):
        infos[k] = [off[0], off[1], arr, layer, sc[0], sc[1], uvset, 0]
    return infos, [a0, a1]


def texture_materials(materials: np.ndarray, seed: int = 0) -> np.ndarray:
    """Copies of the material records with texture references on every texture
    slot over the set (each material gets about half of the slots)."""
    rng = np.random.default_rng(seed)
    out = np.array(materials, np.float32, copy=True)
    fixed = {"baseColorTextureId": 0, "metallicRoughnessTextureId": 1, "normalTextureId": 2, "emissiveTextureId": 3,
             "specularColorTextureId": 5, "anisotropyDirectionTextureId": 6, "sheenColorTextureId": 8}
    for m in range(out.shape[0]):
        for slot in TEXTURE_SLOTS:
            if rng.uniform() < 0.5:
                tid = fixed.get(slot, int(rng.integers(0, 9)))
                out[m, MAT[slot]] = tid
        out[m, MAT["emissiveFactor"]:MAT["emissiveFactor"] + 3] = np.maximum(
            out[m, MAT["emissiveFactor"]:MAT["emissiveFactor"] + 3], 0.5 if rng.uniform() < 0.25 else 0.0)
    return out


def make_textured_small(seed: int = 0) -> Scene:
    """The small scene with planar uvs on every vertex and textured materials."""
    sc = make_small(seed)
    v = sc.vertices.copy()
    p = v[:, 0:3]
    v[:, 8] = p[:, 0] * 0.9 + p[:, 1] * 0.35
    v[:, 9] = p[:, 2] * 0.8 + p[:, 1] * 0.55
    sc.vertices = v
    sc.materials = texture_materials(sc.materials, seed + 1)
    sc.name = "small-textured"
    sc.tex_infos, sc.tex_arrays = texture_set(seed + 2)
    return sc


WORKLOADS = {"small": make_small, "large": make_large, "large_framed": make_large_framed,
             "divergence": make_divergence}


# ---- request mixes of the batching / serving configurations ----------------
def scene_set(seed: int, n: int, lo_tris: int, hi_tris: int, env_size=(1024, 512)) -> list[Scene]:
    """n resident scenes with log-uniform triangle counts in [lo_tris, hi_tris]
    (endpoints included), generated like the large configuration."""
    rng = np.random.default_rng(seed)
    counts = np.exp(np.linspace(np.log(lo_tris), np.log(hi_tris), n))
    rng.shuffle(counts)
    return [make_sized(seed * 1000 + k, int(c), env_size) for k, c in enumerate(counts)]


def request_mix(seed: int, n: int, n_scenes: int, px_lo: int, px_hi: int, spp_lo: int, spp_hi: int,
                fov_lo: float = 30.0, fov_hi: float = 90.0, max_bounces: int = 12, aspect_hi: float = 1.0) -> list[dict]:
    """n viewport requests: scene index, random camera around the 100 m
    instance cube, pixel count log-uniform in [px_lo, px_hi] (aspect ratio
    uniform in [1, aspect_hi]), spp uniform in [spp_lo, spp_hi], fov uniform."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        npx = float(np.exp(rng.uniform(np.log(px_lo), np.log(px_hi))))
        a = float(rng.uniform(1.0, aspect_hi))
        w = max(1, int(round(np.sqrt(npx * a))))
        h = max(1, int(round(npx / w)))
        d = rng.normal(size=3)
        d[1] = abs(d[1]) + 0.2
        d /= np.linalg.norm(d)
        pos = d * rng.uniform(110.0, 170.0)
        target = rng.uniform(-25.0, 25.0, 3)
        fov = float(rng.uniform(fov_lo, fov_hi))
        cam = Camera.look_at(pos, target, fov=fov, near=0.1)
        out.append({"scene": int(rng.integers(0, n_scenes)), "camera": cam, "width": w, "height": h,
                    "spp": int(rng.integers(spp_lo, spp_hi + 1)), "maxBounces": max_bounces})
    return out
