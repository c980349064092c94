"""glTF 2.0 scene packing: a .gltf / .glb file to the reference's scene buffers.

Restates the reference loader (packages/lib/loaders/scene_loader.ts) on top of
a glTF reader written here.  The reference reads through glTF-Transform 4.3.0
(@gltf-transform/core, /extensions, /functions; yarn.lock:381-405) and decodes
images with the browser; neither is available to a Python host, so the parts
of those libraries the loader relies on are restated from the glTF 2.0
specification:

* containers: .gltf (JSON with external or ``data:`` URI buffers and images)
  and .glb (JSON + BIN chunks);
* accessors: strided buffer views, sparse substitution, and the ``dequantize()``
  transform the loader applies first (scene_loader.ts:42): every vertex
  attribute becomes float32, normalized integers decoded as c/255, c/65535,
  max(c/127, -1), max(c/32767, -1);
* material getters return the glTF defaults (metallicFactor 1, roughness 1,
  alphaCutoff 0.5, ...) and the KHR_materials_* extension defaults;
* a texture is its source image (EXT_texture_webp / EXT_texture_avif sources
  first); TextureInfo carries texCoord and KHR_texture_transform offset/scale.

The packing itself follows the reference step by step:

* traversal (scene_loader.ts:175-221): the first scene's root nodes pushed on a
  stack in order and popped from the end; a node's children are pushed before
  its mesh is packed; world = parent x local, with the float32 storage of the
  reference's Float32Array matrices;
* vertices (packPrimitive, :243-344): 20 floats per vertex, world-space
  position + material index, normal by the normal matrix (inverse transpose,
  normalized when longer than 1e-8), uv0, uv1, tangent (xyz by the normal
  matrix, w kept), colour (RGB colours get alpha 1; no colour: white);
  primitives without indices or positions are skipped; the primitive mode is
  not looked at;
* materials (createMaterialData, :348-478): MaterialData defaults
  (material.ts:436-480) overridden by the core fields and each extension;
  material indices in order of first use, 0 for primitives without one;
* textures (ensureTexture / addTexture, scene_data.ts:71-100): ids in order of
  first request within each material (base colour, metallic-roughness,
  normal, emissive, specular, specular colour, transmission, clearcoat,
  clearcoat roughness, clearcoat normal, sheen colour, sheen roughness,
  anisotropy, iridescence, iridescence thickness, diffuse transmission,
  diffuse transmission colour); one TexInfo per distinct (image, colour
  space, uv set, offset, scale); one RGBA8 array per image resolution, one
  layer per distinct (image, colour space);
* with no material at all, one all-zero record (scene_data_webgl2.ts:144-149);
  with no texture, the reference's default TexInfo (array 255: white).

Deliberate differences, each documented where it applies: node matrices are
used as given (the reference round-trips them through translation / rotation /
scale in glTF-Transform, equal up to rounding for the TRS matrices the spec
allows); images are decoded with Pillow into straight RGBA8 (the browser's
canvas round trip through premultiplied alpha can change the RGB of
translucent texels); meshopt- and Draco-compressed files are refused.
"""
from __future__ import annotations

import base64
import hashlib
import io
import json
import math
import os
import struct

import numpy as np

from . import synth
from .synth import MATERIAL_STRIDE, VERTEX_STRIDE

_DTYPES = {5120: np.int8, 5121: np.uint8, 5122: np.int16, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_NCOMP = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT2": 4, "MAT3": 9, "MAT4": 16}
_NORMALIZE = {5121: (255.0, None), 5123: (65535.0, None), 5120: (127.0, -1.0), 5122: (32767.0, -1.0)}
_SUPPORTED_MIME = {"image/png", "image/jpeg", "image/webp", "image/avif"}
_EXT_MIME = {".png": "image/png", ".jpg": "image/jpeg", ".jpeg": "image/jpeg", ".webp": "image/webp",
             ".avif": "image/avif", ".ktx2": "image/ktx2"}
# extensions this reader understands (anything else listed in extensionsRequired is refused)
_KNOWN_EXTENSIONS = {
    "KHR_materials_emissive_strength", "KHR_materials_ior", "KHR_materials_specular",
    "KHR_materials_transmission", "KHR_materials_volume", "KHR_materials_clearcoat", "KHR_materials_sheen",
    "KHR_materials_anisotropy", "KHR_materials_iridescence", "KHR_materials_dispersion",
    "KHR_materials_diffuse_transmission", "KHR_texture_transform", "KHR_mesh_quantization",
    "KHR_lights_punctual", "EXT_texture_webp", "EXT_texture_avif", "KHR_materials_unlit",
    "KHR_materials_variants", "KHR_xmp_json_ld",
}
_COMPRESSION = {"EXT_meshopt_compression", "KHR_meshopt_compression", "KHR_draco_mesh_compression"}

# the reference's default TexInfo when a scene has no texture (scene_data_webgl2.ts:313-315)
DEFAULT_TEX_INFO = np.array([0, 0, 255, 255, 1, 1, 255, 0], np.float32)


class GltfError(ValueError):
    pass


# ---- container -------------------------------------------------------------------------------
class _Document:
    def __init__(self, gltf: dict, buffers: list[bytes], base_dir: str | None):
        self.j = gltf
        self.buffers = buffers
        self.base_dir = base_dir
        self._acc_cache: dict[tuple, np.ndarray] = {}
        self._img_cache: dict[int, tuple[bytes, str]] = {}

    def list(self, key):
        return self.j.get(key, []) or []

    # -- buffers --
    def view_bytes(self, bv_index: int) -> tuple[memoryview, int]:
        bv = self.list("bufferViews")[bv_index]
        if any(e in (bv.get("extensions") or {}) for e in _COMPRESSION):
            raise GltfError("compressed buffer views (EXT_meshopt_compression) are not supported")
        buf = self.buffers[bv["buffer"]]
        off = int(bv.get("byteOffset", 0))
        n = int(bv["byteLength"])
        if off + n > len(buf):
            raise GltfError(f"bufferView {bv_index} overruns its buffer")
        return memoryview(buf)[off:off + n], int(bv.get("byteStride", 0) or 0)

    # -- accessors (glTF 2.0 section 3.6) --
    def _raw(self, bv_index, byte_offset, ctype, ncomp, count, stride_hint=True) -> np.ndarray:
        dt = np.dtype(_DTYPES[ctype]).newbyteorder("<")
        data, stride = self.view_bytes(bv_index)
        elem = dt.itemsize * ncomp
        stride = stride if (stride and stride_hint) else elem
        if count == 0:
            return np.zeros((0, ncomp), dt)
        need = byte_offset + stride * (count - 1) + elem
        if need > len(data):
            raise GltfError("accessor overruns its bufferView")
        a = np.ndarray((count, ncomp), dt, buffer=data, offset=byte_offset, strides=(stride, dt.itemsize))
        return np.array(a, dt.newbyteorder("="))

    def accessor(self, index: int) -> tuple[np.ndarray, dict]:
        """(count, ncomp) array in the accessor's component type, sparse values applied."""
        acc = self.list("accessors")[index]
        ctype = int(acc["componentType"])
        if ctype not in _DTYPES:
            raise GltfError(f"accessor {index}: component type {ctype}")
        ncomp = _NCOMP[acc["type"]]
        count = int(acc["count"])
        if "bufferView" in acc:
            a = self._raw(acc["bufferView"], int(acc.get("byteOffset", 0)), ctype, ncomp, count)
        else:
            a = np.zeros((count, ncomp), _DTYPES[ctype])
        sp = acc.get("sparse")
        if sp:
            n = int(sp["count"])
            ii = sp["indices"]
            idx = self._raw(ii["bufferView"], int(ii.get("byteOffset", 0)), int(ii["componentType"]), 1, n,
                            stride_hint=False)[:, 0].astype(np.int64)
            vv = sp["values"]
            vals = self._raw(vv["bufferView"], int(vv.get("byteOffset", 0)), ctype, ncomp, n, stride_hint=False)
            if n and (idx.min() < 0 or idx.max() >= count):
                raise GltfError(f"accessor {index}: sparse index out of range")
            a = a.copy()
            a[idx] = vals
        return a, acc

    def attribute_f32(self, index: int) -> np.ndarray:
        """An attribute after glTF-Transform's dequantize(): float32, normalized
        integers decoded (MathUtils.decodeNormalizedInt)."""
        key = ("f32", index)
        if key not in self._acc_cache:
            a, acc = self.accessor(index)
            ctype = int(acc["componentType"])
            if ctype == 5126:
                out = a.astype(np.float32)
            elif acc.get("normalized", False):
                div, lo = _NORMALIZE.get(ctype, (1.0, None))
                x = a.astype(np.float64) / div
                if lo is not None:
                    x = np.maximum(x, lo)
                out = x.astype(np.float32)
            else:
                out = a.astype(np.float32)
            self._acc_cache[key] = out
        return self._acc_cache[key]

    def indices_u32(self, index: int) -> np.ndarray:
        a, _ = self.accessor(index)
        return a.reshape(-1).astype(np.uint32)

    # -- images --
    def image(self, index: int) -> tuple[bytes, str, str]:
        """(bytes, mime type, name) of images[index]."""
        img = self.list("images")[index]
        name = img.get("name", "") or ""
        if index in self._img_cache:
            b, mime = self._img_cache[index]
            return b, mime, name
        mime = img.get("mimeType", "")
        if "bufferView" in img:
            data, _ = self.view_bytes(img["bufferView"])
            b = bytes(data)
        elif "uri" in img:
            b, m = self._uri(img["uri"])
            mime = mime or m
        else:
            b = b""
        self._img_cache[index] = (b, mime)
        return b, mime, name

    def _uri(self, uri: str) -> tuple[bytes, str]:
        if uri.startswith("data:"):
            head, _, payload = uri.partition(",")
            mime = head[5:].split(";")[0]
            return (base64.b64decode(payload) if ";base64" in head else payload.encode()), mime
        if self.base_dir is None:
            raise GltfError(f"external resource {uri!r} without a base directory")
        from urllib.parse import unquote
        path = os.path.join(self.base_dir, unquote(uri))
        with open(path, "rb") as f:
            b = f.read()
        return b, _EXT_MIME.get(os.path.splitext(path)[1].lower(), "")


def _read_container(source, resources: dict | None = None) -> _Document:
    base_dir = None
    if isinstance(source, (str, os.PathLike)):
        base_dir = os.path.dirname(os.path.abspath(source))
        with open(source, "rb") as f:
            raw = f.read()
    else:
        raw = bytes(source)
    bin_chunk = None
    if raw[:4] == b"glTF":
        version, length = struct.unpack_from("<II", raw, 4)
        if version != 2:
            raise GltfError(f"GLB version {version}")
        off, js = 12, None
        while off + 8 <= min(length, len(raw)):
            clen, ctype = struct.unpack_from("<II", raw, off)
            body = raw[off + 8:off + 8 + clen]
            if ctype == 0x4E4F534A:
                js = json.loads(body.decode("utf-8"))
            elif ctype == 0x004E4942 and bin_chunk is None:
                bin_chunk = body
            off += 8 + clen
        if js is None:
            raise GltfError("GLB without a JSON chunk")
    else:
        js = json.loads(raw.decode("utf-8"))
    req = set(js.get("extensionsRequired", []) or [])
    bad = sorted(req & _COMPRESSION)
    if bad:
        raise GltfError(f"compressed geometry ({', '.join(bad)}) is not supported")
    unknown = sorted(req - _KNOWN_EXTENSIONS)
    if unknown:
        raise GltfError(f"required extensions not supported: {', '.join(unknown)}")
    doc = _Document(js, [], base_dir)
    buffers = []
    for k, b in enumerate(js.get("buffers", []) or []):
        uri = b.get("uri")
        if uri is None:
            if bin_chunk is None:
                raise GltfError(f"buffer {k} has no uri and the file has no BIN chunk")
            buffers.append(bin_chunk)
        elif resources is not None and uri in resources:
            buffers.append(bytes(resources[uri]))
        else:
            buffers.append(doc._uri(uri)[0])
    doc.buffers = buffers
    return doc


# ---- matrices (float32 storage, float64 arithmetic, as the reference's Float32Array math) -----
def _trs_matrix(node: dict) -> np.ndarray:
    """nodeToMatrix (scene_loader.ts:553-570): column-major TRS composition."""
    t = node.get("translation", [0, 0, 0])
    qx, qy, qz, qw = node.get("rotation", [0, 0, 0, 1])
    sx, sy, sz = node.get("scale", [1, 1, 1])
    x2, y2, z2 = qx * 2, qy * 2, qz * 2
    xx, xy, xz = qx * x2, qx * y2, qx * z2
    yy, yz, zz = qy * y2, qy * z2, qz * z2
    wx, wy, wz = qw * x2, qw * y2, qw * z2
    m = np.zeros(16, np.float64)
    m[0], m[1], m[2] = (1 - (yy + zz)) * sx, (xy + wz) * sx, (xz - wy) * sx
    m[4], m[5], m[6] = (xy - wz) * sy, (1 - (xx + zz)) * sy, (yz + wx) * sy
    m[8], m[9], m[10] = (xz + wy) * sz, (yz - wx) * sz, (1 - (xx + yy)) * sz
    m[12], m[13], m[14], m[15] = t[0], t[1], t[2], 1
    return m.astype(np.float32)


def _local_matrix(node: dict) -> np.ndarray:
    if "matrix" in node:
        return np.asarray(node["matrix"], np.float64).astype(np.float32)
    return _trs_matrix(node)


def _mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """multiplyMat4 (scene_loader.ts:572-582): float64 sums over k in order, stored as float32."""
    a64, b64 = a.astype(np.float64), b.astype(np.float64)
    out = np.zeros(16, np.float64)
    for row in range(4):
        for col in range(4):
            s = 0.0
            for k in range(4):
                s += a64[row + k * 4] * b64[k + col * 4]
            out[row + col * 4] = s
    return out.astype(np.float32)


def _normal_matrix(w: np.ndarray) -> np.ndarray:
    """getNormalMatrix (scene_loader.ts:584-600): inverse transpose of the upper 3x3."""
    e = w.astype(np.float64)
    a00, a01, a02 = e[0], e[4], e[8]
    a10, a11, a12 = e[1], e[5], e[9]
    a20, a21, a22 = e[2], e[6], e[10]
    b01 = a22 * a11 - a12 * a21
    b11 = -a22 * a10 + a12 * a20
    b21 = a21 * a10 - a11 * a20
    det = a00 * b01 + a01 * b11 + a02 * b21
    if abs(det) <= 1e-12:
        return np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    det = 1 / det
    return np.array([b01 * det, (-a22 * a01 + a02 * a21) * det, (a12 * a01 - a02 * a11) * det,
                     b11 * det, (a22 * a00 - a02 * a20) * det, (-a12 * a00 + a02 * a10) * det,
                     b21 * det, (-a21 * a00 + a01 * a20) * det, (a11 * a00 - a01 * a10) * det], np.float32)


def _transform_points(p: np.ndarray, m: np.ndarray) -> np.ndarray:
    """transformPoint (scene_loader.ts:602-608), vectorised, same operation order."""
    m = m.astype(np.float64)
    x, y, z = (p[:, k].astype(np.float64) for k in range(3))
    out = np.empty((p.shape[0], 3), np.float32)
    out[:, 0] = m[0] * x + m[4] * y + m[8] * z + m[12]
    out[:, 1] = m[1] * x + m[5] * y + m[9] * z + m[13]
    out[:, 2] = m[2] * x + m[6] * y + m[10] * z + m[14]
    return out


def _transform_dirs(d: np.ndarray, n: np.ndarray) -> np.ndarray:
    """transformDir (scene_loader.ts:610-616): normal matrix, then normalise when longer than 1e-8."""
    n = n.astype(np.float64)
    x, y, z = (d[:, k].astype(np.float64) for k in range(3))
    rx = n[0] * x + n[3] * y + n[6] * z
    ry = n[1] * x + n[4] * y + n[7] * z
    rz = n[2] * x + n[5] * y + n[8] * z
    ln = np.sqrt(rx * rx + ry * ry + rz * rz)
    ok = ln > 1e-8
    inv = np.where(ok, 1.0 / np.where(ok, ln, 1.0), 1.0)
    return np.stack([np.where(ok, rx * inv, rx), np.where(ok, ry * inv, ry), np.where(ok, rz * inv, rz)],
                    1).astype(np.float32)


# ---- textures ----------------------------------------------------------------------------------
def decode_image(data: bytes, mime: str) -> np.ndarray:
    """RGBA8 (h, w, 4), row 0 = the image's first (top) row, as getImageData returns it."""
    try:
        from PIL import Image, ImageOps
    except ImportError as e:  # pragma: no cover - Pillow is part of the image
        raise GltfError("decoding textures needs Pillow") from e
    im = Image.open(io.BytesIO(data))
    im = ImageOps.exif_transpose(im)  # createImageBitmap's default image orientation
    if im.mode in ("I;16", "I;16B", "I;16L", "I"):
        a = (np.asarray(im, np.uint32) >> 8).astype(np.uint8)  # high byte, as 16-bit RGB decodes
        rgba = np.empty(a.shape + (4,), np.uint8)
        rgba[..., 0] = rgba[..., 1] = rgba[..., 2] = a
        rgba[..., 3] = 255
        return rgba
    return np.ascontiguousarray(np.asarray(im.convert("RGBA"), np.uint8))


def _texture_image_index(doc: _Document, tex_index: int) -> int | None:
    t = doc.list("textures")[tex_index]
    ext = t.get("extensions") or {}
    for name in ("EXT_texture_webp", "EXT_texture_avif", "KHR_texture_basisu"):
        if name in ext and "source" in ext[name]:
            return int(ext[name]["source"])
    return int(t["source"]) if "source" in t else None


class _TextureTable:
    """PathtracingSceneData.addTexture (scene_data.ts:71-100) + the loader's
    texture cache (scene_loader.ts:109-122, 480-551)."""

    def __init__(self, doc: _Document):
        self.doc = doc
        self.infos: list[np.ndarray] = []
        self.arrays: dict[tuple[int, int], list[tuple[tuple, np.ndarray]]] = {}  # (w, h) -> [(uuid, rgba)]
        self.cache: dict[tuple, int] = {}
        self._decoded: dict[tuple, np.ndarray] = {}

    def ensure(self, info: dict | None, color_space: str) -> int:
        if not info or "index" not in info:
            return -1
        img_index = _texture_image_index(self.doc, int(info["index"]))
        if img_index is None:
            return -1
        data, mime, name = self.doc.image(img_index)
        if not mime and data:
            mime = _sniff_mime(data)
        digest = hashlib.sha256(data).hexdigest() if data else "noimage"
        tr = (info.get("extensions") or {}).get("KHR_texture_transform") or {}
        offset = tuple(float(x) for x in tr.get("offset", [0.0, 0.0]))
        scale = tuple(float(x) for x in tr.get("scale", [1.0, 1.0]))
        uv_set = int(info.get("texCoord", 0))
        key = (name, mime, color_space, digest, uv_set, offset, scale)
        if key in self.cache:
            return self.cache[key]
        if not data or mime not in _SUPPORTED_MIME:
            raise GltfError(f'Unsupported texture "{name}" ({mime or "unknown mime"})')
        dkey = (digest, mime)
        if dkey not in self._decoded:
            self._decoded[dkey] = decode_image(data, mime)
        rgba = self._decoded[dkey]
        h, w = rgba.shape[:2]
        uuid = (name, mime, color_space, w, h, digest)
        res = (w, h)
        rec = np.zeros(8, np.float32)
        if res in self.arrays:
            layers = self.arrays[res]
            layer = next((k for k, (u, _) in enumerate(layers) if u == uuid), -1)
            if layer < 0:
                layers.append((uuid, rgba))
                layer = len(layers) - 1
            rec[2] = list(self.arrays).index(res)
            rec[3] = layer
        else:
            self.arrays[res] = [(uuid, rgba)]
            rec[2] = len(self.arrays) - 1
            rec[3] = 0
        rec[0:2] = offset
        rec[4:6] = scale
        rec[6] = uv_set
        self.infos.append(rec)
        self.cache[key] = len(self.infos) - 1
        return self.cache[key]

    def packed(self) -> tuple[np.ndarray, list[np.ndarray]]:
        if not self.infos:
            return DEFAULT_TEX_INFO.reshape(1, 8).copy(), []
        arrays = [np.stack([rgba for _, rgba in layers]) for layers in self.arrays.values()]
        return np.stack(self.infos), arrays


def _sniff_mime(b: bytes) -> str:
    if b[:8] == b"\x89PNG\r\n\x1a\n":
        return "image/png"
    if b[:3] == b"\xff\xd8\xff":
        return "image/jpeg"
    if b[:4] == b"RIFF" and b[8:12] == b"WEBP":
        return "image/webp"
    if b[4:12] in (b"ftypavif", b"ftypavis"):
        return "image/avif"
    return ""


# ---- materials ---------------------------------------------------------------------------------
def _material(doc: _Document, mat: dict, tex: _TextureTable) -> np.ndarray:
    """createMaterialData (scene_loader.ts:348-478) over MaterialData() defaults."""
    m = synth.default_material()
    put = lambda k, v: synth.set_field(m, k, v)  # noqa: E731
    pbr = mat.get("pbrMetallicRoughness") or {}
    bc = pbr.get("baseColorFactor", [1, 1, 1, 1])
    put("baseColorFactor", bc[:3])
    alpha_mode = mat.get("alphaMode", "OPAQUE")
    base_alpha = bc[3] if len(bc) > 3 else 1.0
    put("cutoutOpacity", 1.0 if alpha_mode == "OPAQUE" else base_alpha)
    cutoff = mat.get("alphaCutoff", 0.5) if alpha_mode == "MASK" else (1.0 if alpha_mode == "OPAQUE" else 0.0)
    put("alphaCutoff", cutoff)
    put("metallicFactor", pbr.get("metallicFactor", 1.0))
    put("roughnessFactor", pbr.get("roughnessFactor", 1.0))
    nt = mat.get("normalTexture") or None
    put("normalScale", (nt or {}).get("scale", 1.0))
    emissive = list(mat.get("emissiveFactor", [0, 0, 0]))
    put("doubleSided", 1 if mat.get("doubleSided", False) else 0)
    put("baseColorTextureId", tex.ensure(pbr.get("baseColorTexture"), "srgb"))
    put("metallicRoughnessTextureId", tex.ensure(pbr.get("metallicRoughnessTexture"), "linear"))
    put("normalTextureId", tex.ensure(nt, "linear"))
    put("emissiveTextureId", tex.ensure(mat.get("emissiveTexture"), "srgb"))
    ext = mat.get("extensions") or {}
    e = ext.get("KHR_materials_emissive_strength")
    if e is not None:
        s = e.get("emissiveStrength", 1.0)
        emissive = [c * s for c in emissive]
    put("emissiveFactor", emissive)
    e = ext.get("KHR_materials_ior")
    if e is not None:
        put("ior", e.get("ior", 1.5))
    e = ext.get("KHR_materials_specular")
    if e is not None:
        put("specularFactor", e.get("specularFactor", 1.0))
        put("specularColorFactor", e.get("specularColorFactor", [1, 1, 1]))
        put("specularTextureId", tex.ensure(e.get("specularTexture"), "linear"))
        put("specularColorTextureId", tex.ensure(e.get("specularColorTexture"), "srgb"))
    e = ext.get("KHR_materials_transmission")
    if e is not None:
        put("transmissionFactor", e.get("transmissionFactor", 0.0))
        put("transmissionTextureId", tex.ensure(e.get("transmissionTexture"), "linear"))
    e = ext.get("KHR_materials_volume")
    if e is not None:
        put("thinWalled", 1 if e.get("thicknessFactor", 0.0) == 0 else 0)
        put("attenuationColor", e.get("attenuationColor", [1, 1, 1]))
        dist = e.get("attenuationDistance", math.inf)
        put("attenuationDistance", math.inf if (not dist or dist == 0) else dist)  # MAX_VALUE -> float32 inf
    e = ext.get("KHR_materials_clearcoat")
    if e is not None:
        put("clearcoatFactor", e.get("clearcoatFactor", 0.0))
        put("clearcoatRoughnessFactor", e.get("clearcoatRoughnessFactor", 0.0))
        cn = e.get("clearcoatNormalTexture") or None
        put("clearcoatNormalTextureScale", (cn or {}).get("scale", 1.0))
        put("clearcoatTextureId", tex.ensure(e.get("clearcoatTexture"), "linear"))
        put("clearcoatRoughnessTextureId", tex.ensure(e.get("clearcoatRoughnessTexture"), "linear"))
        put("clearcoatNormalTextureId", tex.ensure(cn, "linear"))
    e = ext.get("KHR_materials_sheen")
    if e is not None:
        put("sheenColorFactor", e.get("sheenColorFactor", [0, 0, 0]))
        put("sheenRoughnessFactor", e.get("sheenRoughnessFactor", 0.0))
        put("sheenColorTextureId", tex.ensure(e.get("sheenColorTexture"), "srgb"))
        put("sheenRoughnessTextureId", tex.ensure(e.get("sheenRoughnessTexture"), "linear"))
    e = ext.get("KHR_materials_anisotropy")
    if e is not None:
        rot = e.get("anisotropyRotation", 0.0)
        put("anisotropy", e.get("anisotropyStrength", 0.0))
        put("anisotropyDirection", [math.cos(rot), math.sin(rot), 0.0])
        put("anisotropyTextureId", tex.ensure(e.get("anisotropyTexture"), "linear"))
    e = ext.get("KHR_materials_iridescence")
    if e is not None:
        put("iridescenceFactor", e.get("iridescenceFactor", 0.0))
        put("iridescenceIor", e.get("iridescenceIor", 1.3))
        put("iridescenceThicknessMinimum", e.get("iridescenceThicknessMinimum", 100.0))
        put("iridescenceThicknessMaximum", e.get("iridescenceThicknessMaximum", 400.0))
        put("iridescenceTextureId", tex.ensure(e.get("iridescenceTexture"), "linear"))
        put("iridescenceThicknessTextureId", tex.ensure(e.get("iridescenceThicknessTexture"), "linear"))
    e = ext.get("KHR_materials_dispersion")
    if e is not None:
        put("dispersion", e.get("dispersion", 0.0))
    e = ext.get("KHR_materials_diffuse_transmission")
    if e is not None:
        put("diffuseTransmissionFactor", e.get("diffuseTransmissionFactor", 0.0))
        put("diffuseTransmissionColorFactor", e.get("diffuseTransmissionColorFactor", [1, 1, 1]))
        put("diffuseTransmissionTextureId", tex.ensure(e.get("diffuseTransmissionTexture"), "linear"))
        put("diffuseTransmissionColorTextureId", tex.ensure(e.get("diffuseTransmissionColorTexture"), "srgb"))
    return m


# ---- scene ----------------------------------------------------------------------------------------
def _pack_primitive(doc: _Document, prim: dict, world: np.ndarray, nrm_m: np.ndarray, mat_idx: int):
    """packPrimitive (scene_loader.ts:243-344): (vertices (V, 20), local indices) or None."""
    attrs = prim.get("attributes", {})
    if "indices" not in prim or "POSITION" not in attrs:
        return None
    if any(e in (prim.get("extensions") or {}) for e in _COMPRESSION):
        raise GltfError("compressed primitives (KHR_draco_mesh_compression) are not supported")
    pos = doc.attribute_f32(attrs["POSITION"])
    n = pos.shape[0]
    idx = doc.indices_u32(prim["indices"])
    v = np.zeros((n, VERTEX_STRIDE), np.float32)
    v[:, 0:3] = _transform_points(pos, world)
    v[:, 3] = mat_idx
    for key in ("NORMAL", "TANGENT"):
        if key in attrs and doc.attribute_f32(attrs[key]).shape[0] != n:
            raise GltfError(f"{key} count differs from POSITION count")
    if "NORMAL" in attrs:
        v[:, 4:7] = _transform_dirs(doc.attribute_f32(attrs["NORMAL"]), nrm_m)
    for slot, key in ((8, "TEXCOORD_0"), (10, "TEXCOORD_1")):
        if key in attrs:
            uv = doc.attribute_f32(attrs[key])
            k = min(n, uv.shape[0])
            v[:k, slot:slot + 2] = uv[:k, :2]
    if "TANGENT" in attrs:
        t = doc.attribute_f32(attrs["TANGENT"])
        v[:, 12:15] = _transform_dirs(t, nrm_m)
        v[:, 15] = t[:, 3]
    v[:, 16:20] = 1.0
    if "COLOR_0" in attrs:
        c = doc.attribute_f32(attrs["COLOR_0"])
        k = min(n, c.shape[0])
        v[:k, 16:16 + min(c.shape[1], 4)] = c[:k, :4]
        if c.shape[1] == 3:
            v[:k, 19] = 1.0
    return v, idx


def load_gltf(source, resources: dict | None = None, punctual_lights: bool = False,
              name: str | None = None) -> synth.Scene:
    """Packs a glTF 2.0 asset (path to .gltf / .glb, or its bytes) into a
    synth.Scene: vertices (V, 20), indices, materials (M, 68), tex_infos
    (N, 8) + tex_arrays [(layers, h, w, 4) uint8], lights.

    ``resources`` maps buffer / image URIs to bytes for in-memory assets.
    ``punctual_lights``: the reference asks the node for ``getLight()``, which
    glTF-Transform 4.3's Node does not have, so its scenes never get a light;
    True adds KHR_lights_punctual lights of mesh nodes as that code intends
    (position = world translation, type 0 point / 1 other, emission = colour x
    intensity).  The camera frames the scene's bounds (the reference's loader
    has none; the app places it).
    """
    doc = _read_container(source, resources)
    scenes = doc.list("scenes")
    if not scenes:
        raise GltfError("This model contains no scene.")
    nodes = doc.list("nodes")
    meshes = doc.list("meshes")
    lights_def = ((doc.j.get("extensions") or {}).get("KHR_lights_punctual") or {}).get("lights", [])
    tex = _TextureTable(doc)
    materials: list[np.ndarray] = []
    mat_cache: dict[int, int] = {}
    verts, idxs, lights = [], [], []
    offset = 0
    stack = [(int(n), np.eye(4, dtype=np.float32).reshape(16)) for n in scenes[0].get("nodes", [])]
    visited = 0
    while stack:
        ni, parent = stack.pop()
        visited += 1
        if visited > 4 * max(1, len(nodes)) + 16:
            raise GltfError("node graph has a cycle")
        node = nodes[ni]
        world = _mul(parent, _local_matrix(node))
        for c in node.get("children", []):
            stack.append((int(c), world))
        if "mesh" not in node:
            continue
        li = ((node.get("extensions") or {}).get("KHR_lights_punctual") or {}).get("light")
        if punctual_lights and li is not None and 0 <= int(li) < len(lights_def):
            L = lights_def[int(li)]
            col, inten = L.get("color", [1, 1, 1]), L.get("intensity", 1.0)
            lights.append({"position": tuple(float(x) for x in world[12:15]),
                           "type": 0 if L.get("type") == "point" else 1,
                           "emission": tuple(float(c) * inten for c in col)})
        nrm_m = _normal_matrix(world)
        for prim in meshes[int(node["mesh"])].get("primitives", []):
            mi = prim.get("material")
            if mi is None:
                mat_idx = 0
            else:
                mi = int(mi)
                if mi not in mat_cache:
                    materials.append(_material(doc, doc.list("materials")[mi], tex))
                    mat_cache[mi] = len(materials) - 1
                mat_idx = mat_cache[mi]
            packed = _pack_primitive(doc, prim, world, nrm_m, mat_idx)
            if packed is None:
                continue
            v, ix = packed
            if ix.size and int(ix.max()) >= v.shape[0]:
                raise GltfError("primitive index beyond its vertex count")
            verts.append(v)
            idxs.append(ix.astype(np.uint64) + offset)
            offset += v.shape[0]
    if not verts:
        raise GltfError("the scene has no indexed triangle geometry")
    vertices = np.concatenate(verts)
    indices = np.concatenate(idxs)
    if indices.max(initial=0) >= 2 ** 32:
        raise GltfError("more than 2^32 vertices")
    indices = indices.astype(np.uint32)
    mats = np.stack(materials) if materials else np.zeros((1, MATERIAL_STRIDE), np.float32)
    infos, arrays = tex.packed()
    lo, hi = vertices[:, :3].min(0).astype(np.float64), vertices[:, :3].max(0).astype(np.float64)
    c = 0.5 * (lo + hi)
    r = max(float(np.linalg.norm(hi - lo)) * 0.5, 1e-3)
    cam = synth.Camera.look_at(c + np.array([0.0, 0.25 * r, 2.6 * r]), c, fov=45.0, near=max(r * 1e-3, 1e-4))
    sc = synth.Scene(name or "gltf", vertices, indices, mats, cam, 512, 512, 64, 8, 2, None, 0,
                     meta={"gltf_nodes": len(nodes), "gltf_materials": len(materials)})
    sc.tex_infos, sc.tex_arrays = infos, arrays
    sc.lights = lights
    return sc
