"""glTF packing (dspbr.gltf) on the CPU against the rules of the reference loader
(loaders/scene_loader.ts) restated independently here: traversal order, world
transforms, normal matrix, attribute decoding, material fields and defaults,
texture ids / arrays / TexInfo records, container forms, errors."""
import math

import numpy as np
import pytest

from dspbr import gltf, synth
from dspbr.synth import MAT
from dspbr.gltf_writer import GltfBuilder, png_bytes, quad_grid


def quat_y(deg):
    h = math.radians(deg) / 2
    return [0.0, math.sin(h), 0.0, math.cos(h)]


def trs(t=(0, 0, 0), q=(0, 0, 0, 1), s=(1, 1, 1)):
    """Column-major 4x4 (float64) of translation * rotation * scale."""
    x, y, z, w = q
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    M = np.eye(4)
    M[:3, :3] = R * np.asarray(s, np.float64)[None, :]
    M[:3, 3] = t
    return M


def apply(M, p):
    return (M[:3, :3] @ p.T).T + M[:3, 3]


def apply_normal(M, n):
    N = np.linalg.inv(M[:3, :3]).T
    r = (N @ n.T).T
    return r / np.linalg.norm(r, axis=1, keepdims=True)


TRI = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
TRI_N = np.array([[0, 0, 1], [0, 0.6, 0.8], [0.6, 0, 0.8]], np.float32)


def hierarchy_doc():
    b = GltfBuilder()
    tri = b.mesh([{"attributes": {"POSITION": b.accessor(TRI), "NORMAL": b.accessor(TRI_N)},
                   "indices": b.accessor(np.array([0, 1, 2], np.uint16))}])
    qp, qn, quv, qi = quad_grid(1)
    quad = b.mesh([{"attributes": {"POSITION": b.accessor(qp), "NORMAL": b.accessor(qn)},
                    "indices": b.accessor(qi.astype(np.uint8))}])
    Mb = trs((0.5, -1, 2), quat_y(30), (1, 1, 1))
    n_a = b.node(mesh=tri, translation=[0, 1, 0])
    n_b = b.node(mesh=quad, matrix=Mb.T.reshape(-1).tolist())
    root0 = b.node(children=[n_a, n_b], translation=[1, 2, 3], rotation=quat_y(90), scale=[2, 1, 1])
    root1 = b.node(mesh=tri, scale=[1, 2, 3])
    b.scene([root0, root1])
    b.scene([root1])  # a second scene is ignored (listScenes()[0])
    R0 = trs((1, 2, 3), quat_y(90), (2, 1, 1))
    expected = [  # stack order: root1, then root0's children last-first
        (trs(s=(1, 2, 3)), TRI, TRI_N, 3),
        (R0 @ Mb, qp, qn, 4),
        (R0 @ trs((0, 1, 0)), TRI, TRI_N, 3),
    ]
    return b, expected


def test_traversal_order_world_transforms_and_normals():
    b, expected = hierarchy_doc()
    js, res = b.gltf_bytes()
    sc = gltf.load_gltf(js, res)
    v = sc.vertices
    assert v.shape == (10, 20) and v.dtype == np.float32
    off = 0
    for M, p, n, cnt in expected:
        np.testing.assert_allclose(v[off:off + cnt, 0:3], apply(M, p.astype(np.float64)), rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(v[off:off + cnt, 4:7], apply_normal(M, n.astype(np.float64)), rtol=1e-5,
                                   atol=1e-6)
        off += cnt
    # indices offset by the vertices packed before each primitive
    np.testing.assert_array_equal(sc.indices, [0, 1, 2, 3, 4, 6, 3, 6, 5, 7, 8, 9])
    assert (v[:, 3] == 0).all() and (v[:, 7] == 0).all()  # no material: index 0; pad 0
    assert (v[:, 16:20] == 1).all() and (v[:, 8:16] == 0).all()  # no colour: white; no uv / tangent
    assert sc.materials.shape == (1, 68) and not sc.materials.any()  # the all-zero record
    np.testing.assert_array_equal(sc.tex_infos, gltf.DEFAULT_TEX_INFO[None])
    assert sc.tex_arrays == []


def test_attribute_decoding_strides_and_sparse():
    b = GltfBuilder()
    pos = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    uv16 = np.array([[0, 0], [65535, 0], [65535, 32768], [12345, 65535]], np.uint16)
    col8 = np.array([[255, 0, 0], [0, 128, 0], [0, 0, 1], [10, 20, 30]], np.uint8)
    nrm8 = np.array([[0, 0, 127], [0, 0, -128], [0, 127, 0], [-127, 0, 0]], np.int8)  # KHR_mesh_quantization
    tan = np.array([[1, 0, 0, -1]] * 4, np.float32)
    uv1 = np.array([[0.25, 0.5]] * 4, np.float32)
    prim = {"attributes": {
        "POSITION": b.accessor(pos, interleave_pad=8, sparse=([2], [[2.0, 2.0, 0.0]])),
        "TEXCOORD_0": b.accessor(uv16, normalized=True), "COLOR_0": b.accessor(col8, normalized=True),
        "NORMAL": b.accessor(nrm8, normalized=True), "TANGENT": b.accessor(tan), "TEXCOORD_1": b.accessor(uv1)},
        "indices": b.accessor(np.array([0, 1, 2, 0, 2, 3], np.uint32))}
    b.node(mesh=b.mesh([prim]))
    b.scene([0])
    sc = gltf.load_gltf(b.glb_bytes())
    v = sc.vertices
    exp_pos = pos.copy()
    exp_pos[2] = [2, 2, 0]  # sparse substitution
    np.testing.assert_array_equal(v[:, 0:3], exp_pos)
    np.testing.assert_array_equal(v[:, 8:10], (uv16.astype(np.float64) / 65535).astype(np.float32))
    np.testing.assert_array_equal(v[:, 10:12], uv1)
    np.testing.assert_array_equal(v[:, 16:19], (col8.astype(np.float64) / 255).astype(np.float32))
    assert (v[:, 19] == 1).all()  # RGB colour: alpha 1
    n = np.maximum(nrm8.astype(np.float64) / 127, -1)
    np.testing.assert_allclose(v[:, 4:7], n / np.linalg.norm(n, axis=1, keepdims=True), atol=1e-7)
    np.testing.assert_array_equal(v[:, 12:16], tan)


def test_material_fields_defaults_and_extensions():
    b = GltfBuilder()
    mats = [
        {},  # glTF defaults
        {"alphaMode": "MASK", "alphaCutoff": 0.3, "pbrMetallicRoughness": {"baseColorFactor": [0.2, 0.4, 0.6, 0.6],
                                                                            "metallicFactor": 0.25,
                                                                            "roughnessFactor": 0.5},
         "doubleSided": True, "normalTexture": None},
        {"alphaMode": "BLEND", "pbrMetallicRoughness": {"baseColorFactor": [1, 1, 1, 0.4]},
         "emissiveFactor": [0.1, 0.2, 0.3],
         "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 5.0},
                        "KHR_materials_ior": {"ior": 1.7},
                        "KHR_materials_specular": {"specularFactor": 0.5, "specularColorFactor": [0.9, 0.8, 0.7]},
                        "KHR_materials_transmission": {"transmissionFactor": 0.75},
                        "KHR_materials_volume": {"thicknessFactor": 0.5, "attenuationDistance": 2.0,
                                                 "attenuationColor": [0.5, 0.6, 0.7]},
                        "KHR_materials_clearcoat": {"clearcoatFactor": 0.8, "clearcoatRoughnessFactor": 0.1},
                        "KHR_materials_sheen": {"sheenColorFactor": [0.3, 0.2, 0.1], "sheenRoughnessFactor": 0.4},
                        "KHR_materials_anisotropy": {"anisotropyStrength": 0.5, "anisotropyRotation": 0.3},
                        "KHR_materials_iridescence": {"iridescenceFactor": 1.0, "iridescenceIor": 1.8,
                                                      "iridescenceThicknessMaximum": 500.0},
                        "KHR_materials_dispersion": {"dispersion": 0.4},
                        "KHR_materials_diffuse_transmission": {"diffuseTransmissionFactor": 0.3,
                                                               "diffuseTransmissionColorFactor": [0.1, 0.9, 0.5]}}},
        {"extensions": {"KHR_materials_volume": {}}},  # thickness 0: thin walled, distance infinite
    ]
    for m in mats:
        b.material({k: v for k, v in m.items() if v is not None})
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    prims = []
    for mi in (2, None, 0, 2, 3, 1):  # first use: 2, (none -> 0), 0, 3, 1
        p = {"attributes": {"POSITION": b.accessor(pos)}, "indices": b.accessor(np.array([0, 1, 2], np.uint32))}
        if mi is not None:
            p["material"] = mi
        prims.append(p)
    b.node(mesh=b.mesh(prims))
    b.scene([0])
    sc = gltf.load_gltf(b.gltf_bytes()[0])
    assert sc.materials.shape == (4, 68)
    np.testing.assert_array_equal(sc.vertices[::3, 3], [0, 0, 1, 0, 2, 3])
    F = lambda m, k, n=1: m[MAT[k]:MAT[k] + n]  # noqa: E731
    d = sc.materials[1]  # glTF {} over MaterialData defaults
    ref = synth.default_material()
    for k in ("ior", "specularFactor", "sheenColorFactor", "iridescenceIor", "attenuationDistance", "thinWalled"):
        np.testing.assert_array_equal(F(d, k, 3 if k.endswith("ColorFactor") else 1),
                                      F(ref, k, 3 if k.endswith("ColorFactor") else 1), err_msg=k)
    assert F(d, "metallicFactor")[0] == 1 and F(d, "roughnessFactor")[0] == 1  # glTF defaults
    assert F(d, "cutoutOpacity")[0] == 1 and F(d, "alphaCutoff")[0] == 1 and F(d, "doubleSided")[0] == 0
    assert F(d, "ior")[0] == np.float32(1.49)  # no KHR_materials_ior: the reference default, not glTF's 1.5
    m = sc.materials[3]  # MASK
    np.testing.assert_array_equal(F(m, "baseColorFactor", 3), np.float32([0.2, 0.4, 0.6]))
    assert F(m, "cutoutOpacity")[0] == np.float32(0.6) and F(m, "alphaCutoff")[0] == np.float32(0.3)
    assert F(m, "metallicFactor")[0] == 0.25 and F(m, "roughnessFactor")[0] == 0.5 and F(m, "doubleSided")[0] == 1
    e = sc.materials[0]  # BLEND + every extension
    assert F(e, "cutoutOpacity")[0] == np.float32(0.4) and F(e, "alphaCutoff")[0] == 0
    np.testing.assert_allclose(F(e, "emissiveFactor", 3), [0.5, 1.0, 1.5], rtol=1e-7)
    assert F(e, "ior")[0] == np.float32(1.7) and F(e, "specularFactor")[0] == 0.5
    np.testing.assert_array_equal(F(e, "specularColorFactor", 3), np.float32([0.9, 0.8, 0.7]))
    assert F(e, "transmissionFactor")[0] == 0.75 and F(e, "thinWalled")[0] == 0
    assert F(e, "attenuationDistance")[0] == 2 and F(e, "clearcoatFactor")[0] == np.float32(0.8)
    np.testing.assert_array_equal(F(e, "attenuationColor", 3), np.float32([0.5, 0.6, 0.7]))
    np.testing.assert_array_equal(F(e, "sheenColorFactor", 3), np.float32([0.3, 0.2, 0.1]))
    np.testing.assert_allclose(F(e, "anisotropyDirection", 3), [math.cos(0.3), math.sin(0.3), 0], rtol=1e-7)
    assert F(e, "anisotropy")[0] == 0.5 and F(e, "iridescenceFactor")[0] == 1
    assert F(e, "iridescenceIor")[0] == np.float32(1.8) and F(e, "iridescenceThicknessMaximum")[0] == 500
    assert F(e, "iridescenceThicknessMinimum")[0] == 100 and F(e, "dispersion")[0] == np.float32(0.4)
    assert F(e, "diffuseTransmissionFactor")[0] == np.float32(0.3)
    v = sc.materials[2]  # volume without thickness
    assert F(v, "thinWalled")[0] == 1 and np.isinf(F(v, "attenuationDistance")[0])
    assert all(F(x, k)[0] == -1 for x in sc.materials for k in MAT if k.endswith("TextureId"))


def textured_doc():
    rng = np.random.default_rng(5)
    img0 = rng.integers(0, 256, (8, 8, 4), dtype=np.uint8)
    img1 = rng.integers(0, 256, (8, 8, 4), dtype=np.uint8)
    img2 = rng.integers(0, 256, (2, 4, 4), dtype=np.uint8)  # 4 wide, 2 high
    b = GltfBuilder()
    i0 = b.image(png_bytes(img0), name="albedo")
    i1 = b.image(png_bytes(img1), embed=False)
    i2 = b.image(png_bytes(img2))
    t0, t1, t2 = b.texture(i0), b.texture(i1), b.texture(i2)
    t0b = b.texture(i0)  # a second texture on the same image
    xf = {"KHR_texture_transform": {"offset": [0.5, 0.25], "scale": [2.0, 3.0]}}
    mA = b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": t0},
                                              "metallicRoughnessTexture": {"index": t0}},
                     "normalTexture": {"index": t2, "scale": 0.5}, "emissiveTexture": {"index": t1}})
    mB = b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": t0b, "texCoord": 1, "extensions": xf}},
                     "extensions": {"KHR_materials_sheen": {"sheenColorTexture": {"index": t2}}}})
    mC = b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": t0b}}})
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    prims = [{"attributes": {"POSITION": b.accessor(pos)}, "indices": b.accessor(np.array([0, 1, 2], np.uint32)),
              "material": mi} for mi in (mA, mB, mC)]
    b.node(mesh=b.mesh(prims))
    b.scene([0])
    return b, (img0, img1, img2)


def test_texture_ids_arrays_and_infos():
    b, (img0, img1, img2) = textured_doc()
    sc = gltf.load_gltf(b.glb_bytes())
    F = lambda m, k: m[MAT[k]]  # noqa: E731
    mA, mB, mC = sc.materials
    # request order in material A: base colour, metallic-roughness, normal, emissive
    assert (F(mA, "baseColorTextureId"), F(mA, "metallicRoughnessTextureId"), F(mA, "normalTextureId"),
            F(mA, "emissiveTextureId")) == (0, 1, 2, 3)
    assert F(mA, "normalScale") == 0.5
    assert (F(mB, "baseColorTextureId"), F(mB, "sheenColorTextureId")) == (4, 5)
    assert F(mC, "baseColorTextureId") == 0  # same image, colour space and transform: the same TexInfo
    infos = sc.tex_infos
    assert infos.shape == (6, 8)
    # (offset.xy, array, layer, scale.xy, uv set, pad)
    np.testing.assert_array_equal(infos[0], [0, 0, 0, 0, 1, 1, 0, 0])   # albedo srgb: 8x8 array, layer 0
    np.testing.assert_array_equal(infos[1], [0, 0, 0, 1, 1, 1, 0, 0])   # albedo linear: a second layer
    np.testing.assert_array_equal(infos[2], [0, 0, 1, 0, 1, 1, 0, 0])   # 4x2 image: second array
    np.testing.assert_array_equal(infos[3], [0, 0, 0, 2, 1, 1, 0, 0])   # emissive image: third 8x8 layer
    np.testing.assert_array_equal(infos[4], [0.5, 0.25, 0, 0, 2, 3, 1, 0])  # transform + uv set 1, layer reused
    np.testing.assert_array_equal(infos[5], [0, 0, 1, 1, 1, 1, 0, 0])   # 4x2 image as srgb: new layer
    a8, a42 = sc.tex_arrays
    assert a8.shape == (3, 8, 8, 4) and a42.shape == (2, 2, 4, 4)
    np.testing.assert_array_equal(a8[0], img0)
    np.testing.assert_array_equal(a8[1], img0)
    np.testing.assert_array_equal(a8[2], img1)
    np.testing.assert_array_equal(a42[0], img2)


def test_containers_agree(tmp_path):
    b, _ = textured_doc()
    ref = gltf.load_gltf(b.glb_bytes())
    js, _ = b.gltf_bytes(data_uri=True)
    others = [gltf.load_gltf(js), gltf.load_gltf(b.write(str(tmp_path / "s.gltf"))),
              gltf.load_gltf(b.write(str(tmp_path / "s.glb")))]
    for o in others:
        np.testing.assert_array_equal(o.vertices, ref.vertices)
        np.testing.assert_array_equal(o.indices, ref.indices)
        np.testing.assert_array_equal(o.materials, ref.materials)
        np.testing.assert_array_equal(o.tex_infos, ref.tex_infos)
        for x, y in zip(o.tex_arrays, ref.tex_arrays):
            np.testing.assert_array_equal(x, y)


def test_lights_and_errors():
    b = GltfBuilder()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    m = b.mesh([{"attributes": {"POSITION": b.accessor(pos)}, "indices": b.accessor(np.array([0, 1, 2], np.uint32))}])
    b.j["extensions"] = {"KHR_lights_punctual": {"lights": [{"type": "spot", "color": [1, 0.5, 0.25],
                                                             "intensity": 4.0}]}}
    b.node(mesh=m, translation=[1, 2, 3], extensions={"KHR_lights_punctual": {"light": 0}})
    b.node(translation=[9, 9, 9], extensions={"KHR_lights_punctual": {"light": 0}})  # no mesh: no light
    b.scene([0, 1])
    js, _ = b.gltf_bytes()
    assert gltf.load_gltf(js).lights == []  # the reference's node.getLight() never answers
    lit = gltf.load_gltf(js, punctual_lights=True).lights
    assert lit == [{"position": (1.0, 2.0, 3.0), "type": 1, "emission": (4.0, 2.0, 1.0)}]
    with pytest.raises(gltf.GltfError):
        gltf.load_gltf(b'{"asset": {"version": "2.0"}}')
    b.j["extensionsRequired"] = ["EXT_meshopt_compression"]
    with pytest.raises(gltf.GltfError):
        gltf.load_gltf(b.gltf_bytes()[0])
    b.j["extensionsRequired"] = []
    b.image(b"\x00\x01", mime="image/ktx2")
    b.material({"pbrMetallicRoughness": {"baseColorTexture": {"index": b.texture(0)}}})
    b.j["meshes"][0]["primitives"][0]["material"] = 0
    with pytest.raises(gltf.GltfError, match="Unsupported texture"):
        gltf.load_gltf(b.gltf_bytes()[0])


def packed_sha(sc) -> bytes:
    import hashlib
    return hashlib.sha256(sc.vertices.tobytes() + sc.indices.tobytes() + sc.materials.tobytes() +
                          sc.tex_infos.tobytes()).digest()


def test_sample_asset_packs_to_the_golden_buffers():
    """The asset the golden glTF image was rendered from still packs to the same bytes."""
    from tests import helpers
    from dspbr.gltf_writer import sample_scene
    g = helpers.load_golden()
    sc = gltf.load_gltf(sample_scene().glb_bytes())
    assert packed_sha(sc) == bytes(g["gltf_vertices_sha"])
    assert sc.vertices.shape == (409, 20) and sc.materials.shape == (4, 68) and len(sc.tex_arrays) == 2
