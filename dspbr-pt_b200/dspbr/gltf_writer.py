"""A small glTF 2.0 writer (glTF 2.0 specification: buffers, buffer views,
accessors, meshes, nodes, materials, images, textures; .gltf with an external
.bin or data: URIs, and .glb).  It makes the seeded synthetic assets that the
loader's tests and the glTF-to-first-frame benchmark read back through
dspbr.gltf.load_gltf."""
from __future__ import annotations

import base64
import io
import json
import os
import struct

import numpy as np

CTYPE = {np.dtype(np.int8): 5120, np.dtype(np.uint8): 5121, np.dtype(np.int16): 5122,
         np.dtype(np.uint16): 5123, np.dtype(np.uint32): 5125, np.dtype(np.float32): 5126}
TYPE = {1: "SCALAR", 2: "VEC2", 3: "VEC3", 4: "VEC4"}


def png_bytes(rgba: np.ndarray) -> bytes:
    from PIL import Image
    b = io.BytesIO()
    a = np.asarray(rgba, np.uint8)
    Image.fromarray(a, "RGBA" if a.shape[-1] == 4 else "RGB").save(b, format="PNG")
    return b.getvalue()


class GltfBuilder:
    def __init__(self):
        self.j = {"asset": {"version": "2.0"}, "buffers": [], "bufferViews": [], "accessors": [], "meshes": [],
                  "nodes": [], "scenes": [], "materials": [], "images": [], "textures": []}
        self.bin = bytearray()

    def _align(self, n=4):
        while len(self.bin) % n:
            self.bin.append(0)

    def view(self, data: bytes, stride: int | None = None) -> int:
        self._align()
        bv = {"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)}
        if stride:
            bv["byteStride"] = stride
        self.bin += data
        self.j["bufferViews"].append(bv)
        return len(self.j["bufferViews"]) - 1

    def accessor(self, a: np.ndarray, normalized: bool = False, interleave_pad: int = 0, minmax: bool = False,
                 sparse: tuple | None = None, no_view: bool = False) -> int:
        a = np.asarray(a)
        if a.ndim == 1:
            a = a[:, None]
        n, k = a.shape
        acc = {"componentType": CTYPE[a.dtype], "count": int(n), "type": TYPE[k]}
        if normalized:
            acc["normalized"] = True
        if not no_view:
            if interleave_pad:
                # strided view: every element followed by interleave_pad bytes of padding
                elem = a.dtype.itemsize * k
                stride = elem + interleave_pad
                stride += (-stride) % 4
                buf = bytearray(stride * n)
                for i in range(n):
                    buf[i * stride:i * stride + elem] = a[i].tobytes()
                acc["bufferView"] = self.view(bytes(buf), stride)
            else:
                acc["bufferView"] = self.view(a.tobytes())
        if minmax:
            acc["min"] = a.min(0).tolist()
            acc["max"] = a.max(0).tolist()
        if sparse is not None:
            idx, vals = sparse
            idx = np.asarray(idx, np.uint32)
            vals = np.asarray(vals, a.dtype).reshape(len(idx), k)
            acc["sparse"] = {"count": int(len(idx)),
                             "indices": {"bufferView": self.view(idx.tobytes()), "componentType": 5125},
                             "values": {"bufferView": self.view(vals.tobytes())}}
        self.j["accessors"].append(acc)
        return len(self.j["accessors"]) - 1

    def mesh(self, primitives: list[dict]) -> int:
        self.j["meshes"].append({"primitives": primitives})
        return len(self.j["meshes"]) - 1

    def node(self, **kw) -> int:
        self.j["nodes"].append(kw)
        return len(self.j["nodes"]) - 1

    def scene(self, roots: list[int]) -> int:
        self.j["scenes"].append({"nodes": roots})
        return len(self.j["scenes"]) - 1

    def material(self, m: dict) -> int:
        self.j["materials"].append(m)
        return len(self.j["materials"]) - 1

    def image(self, data: bytes, mime: str = "image/png", name: str | None = None, embed: bool = True) -> int:
        img = {"mimeType": mime} if embed else {}
        if name:
            img["name"] = name
        if embed:
            img["bufferView"] = self.view(data)
        else:
            img["uri"] = "data:%s;base64,%s" % (mime, base64.b64encode(data).decode())
        self.j["images"].append(img)
        return len(self.j["images"]) - 1

    def texture(self, image: int, ext: dict | None = None) -> int:
        t = {"source": image}
        if ext:
            t["extensions"] = ext
        self.j["textures"].append(t)
        return len(self.j["textures"]) - 1

    def _doc(self, uri: str | None) -> dict:
        j = json.loads(json.dumps(self.j))
        for k in [k for k, v in j.items() if v == [] and k != "scenes"]:
            del j[k]
        self._align()
        buf = {"byteLength": len(self.bin)}
        if uri is not None:
            buf["uri"] = uri
        j["buffers"] = [buf]
        return j

    def gltf_bytes(self, data_uri: bool = True, bin_name: str = "scene.bin") -> tuple[bytes, dict]:
        """(.gltf JSON bytes, resources {uri: bytes})."""
        if data_uri:
            uri = "data:application/octet-stream;base64," + base64.b64encode(bytes(self.bin)).decode()
            return json.dumps(self._doc(uri)).encode(), {}
        return json.dumps(self._doc(bin_name)).encode(), {bin_name: bytes(self.bin)}

    def glb_bytes(self) -> bytes:
        js = json.dumps(self._doc(None)).encode()
        js += b" " * ((-len(js)) % 4)
        b = bytes(self.bin) + b"\0" * ((-len(self.bin)) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(b), 0x004E4942) + b
        return struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body

    def write(self, path: str) -> str:
        if path.endswith(".glb"):
            with open(path, "wb") as f:
                f.write(self.glb_bytes())
        else:
            name = os.path.splitext(os.path.basename(path))[0] + ".bin"
            js, res = self.gltf_bytes(data_uri=False, bin_name=name)
            with open(path, "wb") as f:
                f.write(js)
            with open(os.path.join(os.path.dirname(path), name), "wb") as f:
                f.write(res[name])
        return path


def quad_grid(n: int, size: float = 1.0):
    """(positions, normals, uvs, indices) of an n x n grid in the xy plane."""
    xs = np.linspace(-size, size, n + 1, dtype=np.float32)
    X, Y = np.meshgrid(xs, xs)
    pos = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size, np.float32)], 1).astype(np.float32)
    nrm = np.tile(np.array([0, 0, 1], np.float32), (pos.shape[0], 1))
    uv = np.stack([(X.ravel() + size) / (2 * size), (Y.ravel() + size) / (2 * size)], 1).astype(np.float32)
    idx = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            idx += [a, a + 1, a + n + 2, a, a + n + 2, a + n + 1]
    return pos, nrm, uv, np.asarray(idx, np.uint32)


def sample_scene() -> GltfBuilder:
    """A small seeded glTF asset exercising the loader end to end: a textured
    floor (base colour with alpha, metallic-roughness, normal map, uv
    transform, tangents) under a rotated node, a glass sphere (transmission +
    volume), an iridescent anisotropic sphere with vertex colours, and an
    emissive-textured quad behind them."""
    from dspbr import synth
    rng = np.random.default_rng(11)
    b = GltfBuilder()
    n = 16
    yy, xx = np.mgrid[0:n, 0:n]
    checker = np.zeros((n, n, 4), np.uint8)
    checker[..., :3] = np.where(((xx // 4 + yy // 4) % 2 == 0)[..., None], [200, 180, 150], [40, 60, 90])
    checker[..., 3] = np.where((xx + yy) % 7 == 0, 90, 255)
    orm = rng.integers(0, 256, (n, n, 4), dtype=np.uint8)
    orm[..., 3] = 255
    bump = np.zeros((n, n, 4), np.uint8)
    ang = 2 * np.pi * xx / n
    bump[..., 0] = (127.5 + 80 * np.sin(ang)).astype(np.uint8)
    bump[..., 1] = 128
    bump[..., 2] = (127.5 + 120 * np.abs(np.cos(ang))).astype(np.uint8)
    bump[..., 3] = 255
    glow = np.zeros((8, 8, 4), np.uint8)
    glow[::2, ::2] = [255, 200, 120, 255]
    glow[..., 3] = 255
    t_checker = b.texture(b.image(png_bytes(checker), name="checker"))
    t_orm = b.texture(b.image(png_bytes(orm), name="orm"))
    t_bump = b.texture(b.image(png_bytes(bump), name="bump"))
    t_glow = b.texture(b.image(png_bytes(glow), embed=False))
    xf = {"KHR_texture_transform": {"offset": [0.1, 0.0], "scale": [2.0, 2.0]}}
    m_floor = b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": t_checker, "extensions": xf},
                                                   "metallicRoughnessTexture": {"index": t_orm},
                                                   "metallicFactor": 0.6, "roughnessFactor": 0.9},
                          "normalTexture": {"index": t_bump, "scale": 0.8}, "alphaMode": "MASK",
                          "alphaCutoff": 0.5})
    m_glass = b.material({"pbrMetallicRoughness": {"baseColorFactor": [1, 1, 1, 1], "metallicFactor": 0.0,
                                                   "roughnessFactor": 0.05},
                          "extensions": {"KHR_materials_transmission": {"transmissionFactor": 1.0},
                                         "KHR_materials_volume": {"thicknessFactor": 1.0,
                                                                  "attenuationDistance": 1.5,
                                                                  "attenuationColor": [0.9, 0.6, 0.5]},
                                         "KHR_materials_ior": {"ior": 1.45}}})
    m_irid = b.material({"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.8, 0.8, 1], "metallicFactor": 1.0,
                                                  "roughnessFactor": 0.3},
                         "extensions": {"KHR_materials_iridescence": {"iridescenceFactor": 1.0,
                                                                      "iridescenceThicknessMaximum": 350.0},
                                        "KHR_materials_anisotropy": {"anisotropyStrength": 0.6,
                                                                     "anisotropyRotation": 0.7}}})
    m_emit = b.material({"pbrMetallicRoughness": {"baseColorFactor": [0.1, 0.1, 0.1, 1]},
                         "emissiveFactor": [1.0, 1.0, 1.0], "emissiveTexture": {"index": t_glow},
                         "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 3.0}}})
    # floor: 8x8 grid in xy, rotated to lie in xz
    fp, fn, fuv, fi = quad_grid(8, 2.0)
    ftan = np.tile(np.array([1, 0, 0, 1], np.float32), (fp.shape[0], 1))
    floor = b.mesh([{"attributes": {"POSITION": b.accessor(fp, minmax=True), "NORMAL": b.accessor(fn),
                                    "TEXCOORD_0": b.accessor(fuv), "TANGENT": b.accessor(ftan)},
                     "indices": b.accessor(fi.astype(np.uint16)), "material": m_floor}])
    sv, sf = synth.icosphere(2)
    sv = sv.astype(np.float32)
    col = (0.5 + 0.5 * sv).astype(np.float32)
    stan = np.zeros((sv.shape[0], 4), np.float32)
    stan[:, 0] = -sv[:, 2]
    stan[:, 2] = sv[:, 0]
    stan[:, 3] = 1
    stan[np.abs(stan[:, :3]).sum(1) < 1e-6, 0] = 1
    stan[:, :3] /= np.linalg.norm(stan[:, :3], axis=1, keepdims=True)
    sidx = np.asarray(sf, np.uint32).reshape(-1)
    glass = b.mesh([{"attributes": {"POSITION": b.accessor(sv), "NORMAL": b.accessor(sv)},
                     "indices": b.accessor(sidx), "material": m_glass}])
    irid = b.mesh([{"attributes": {"POSITION": b.accessor(sv), "NORMAL": b.accessor(sv), "TANGENT": b.accessor(stan),
                                   "COLOR_0": b.accessor((col * 255).astype(np.uint8), normalized=True)},
                    "indices": b.accessor(sidx), "material": m_irid}])
    qp, qn, quv, qi = quad_grid(1, 0.6)
    emit = b.mesh([{"attributes": {"POSITION": b.accessor(qp), "NORMAL": b.accessor(qn), "TEXCOORD_0": b.accessor(quv)},
                    "indices": b.accessor(qi), "material": m_emit}])
    n_floor = b.node(mesh=floor, rotation=[-0.7071067811865476, 0, 0, 0.7071067811865476])
    n_glass = b.node(mesh=glass, translation=[-0.6, 0.5, 0.2], scale=[0.45, 0.45, 0.45])
    n_irid = b.node(mesh=irid, translation=[0.7, 0.45, -0.1], scale=[0.4, 0.4, 0.4])
    n_emit = b.node(mesh=emit, translation=[0, 1.0, -1.5])
    group = b.node(children=[n_glass, n_irid], translation=[0, 0.0, 0.0], rotation=[0, 0.0998, 0, 0.995])
    b.scene([n_floor, group, n_emit])
    return b


def sample_camera():
    from dspbr import synth
    return synth.Camera.look_at((0.0, 1.6, 4.2), (0.0, 0.4, 0.0), fov=45.0, near=0.05)


def large_asset(n_nodes: int = 256, seed: int = 0) -> GltfBuilder:
    """~1.9M triangles as glTF instancing: n_nodes nodes over four meshes (a
    9,800-triangle displaced grid and a 5,120-triangle icosphere, twice each,
    with normals, uvs and tangents), four 1024x1024 textures shared by four
    materials, random translation / rotation / scale per node."""
    from dspbr import synth
    rng = np.random.default_rng(seed)
    b = GltfBuilder()
    gp, gn, guv, gi = quad_grid(70, 1.0)
    gp[:, 2] = 0.08 * np.sin(6 * gp[:, 0]) * np.cos(5 * gp[:, 1])
    gtan = np.tile(np.array([1, 0, 0, 1], np.float32), (gp.shape[0], 1))
    sv, sf = synth.icosphere(4)
    sv = sv.astype(np.float32)
    suv = (0.5 + 0.5 * sv[:, :2]).astype(np.float32)
    stan = np.tile(np.array([0, 0, 1, 1], np.float32), (sv.shape[0], 1))
    tex = []
    for k in range(4):
        img = rng.integers(0, 256, (1024, 1024, 4), dtype=np.uint8)
        img[..., 3] = 255
        tex.append(b.texture(b.image(png_bytes(img), name=f"t{k}")))
    mats = []
    for k in range(4):
        mats.append(b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": tex[k]},
                                                         "metallicRoughnessTexture": {"index": tex[(k + 1) % 4]}},
                                "normalTexture": {"index": tex[(k + 2) % 4]},
                                "extensions": {"KHR_materials_clearcoat": {"clearcoatFactor": 0.3 * k}}}))
    meshes = []
    for k in range(4):
        if k % 2 == 0:
            attrs = {"POSITION": b.accessor(gp), "NORMAL": b.accessor(gn), "TEXCOORD_0": b.accessor(guv),
                     "TANGENT": b.accessor(gtan)}
            idx = gi
        else:
            attrs = {"POSITION": b.accessor(sv), "NORMAL": b.accessor(sv), "TEXCOORD_0": b.accessor(suv),
                     "TANGENT": b.accessor(stan)}
            idx = np.asarray(sf, np.uint32).reshape(-1)
        meshes.append(b.mesh([{"attributes": attrs, "indices": b.accessor(idx), "material": mats[k]}]))
    roots = []
    for i in range(n_nodes):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        s = float(rng.uniform(2, 8))
        roots.append(b.node(mesh=meshes[i % 4], translation=rng.uniform(-50, 50, 3).tolist(),
                            rotation=q.tolist(), scale=[s, s, s]))
    b.scene(roots)
    return b
