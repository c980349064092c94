"""Shared inputs for the parity tests (seeded)."""
import numpy as np

from dspbr import synth


def feature_materials(seed=0):
    """One material per DSPBR feature class, plus thin-walled and edge variants."""
    rng = np.random.default_rng(seed)
    mats = [synth.feature_material(rng, k) for k in synth.FEATURES for _ in range(3)]
    m = synth.default_material()  # reference defaults: thin-walled dielectric, roughness 0
    mats.append(m)
    m = synth.feature_material(rng, "transmission")
    synth.set_field(m, "thinWalled", 1.0)
    mats.append(m)
    m = synth.feature_material(rng, "base")
    synth.set_field(m, "diffuseTransmissionFactor", 0.7)
    synth.set_field(m, "diffuseTransmissionColorFactor", [0.8, 0.5, 0.3])
    mats.append(m)
    m = synth.feature_material(rng, "base")
    synth.set_field(m, "specularFactor", 0.0)
    mats.append(m)
    m = synth.glass_material(1.0)  # index matched: null transmission
    mats.append(m)
    return np.stack(mats)


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def bsdf_queries(n, num_materials, seed=1):
    """hit20 / wo3 / rnd4 arrays for dspbr_bsdf_query and the reference harness."""
    rng = np.random.default_rng(seed)
    nrm = unit(rng, n)
    ng = nrm + 0.2 * unit(rng, n)
    ng /= np.linalg.norm(ng, axis=1, keepdims=True)
    tan = unit(rng, n)
    tan -= nrm * np.sum(tan * nrm, axis=1, keepdims=True)
    tan /= np.linalg.norm(tan, axis=1, keepdims=True)
    hand = np.where(rng.uniform(size=n) < 0.5, 1.0, -1.0)
    wi = unit(rng, n)
    wo = unit(rng, n)
    # half the directions on the reflection side of the shading normal
    flip = (rng.uniform(size=n) < 0.5) & (np.sum(wo * nrm, 1) * np.sum(wi * nrm, 1) < 0)
    wo[flip] -= 2 * nrm[flip] * np.sum(wo[flip] * nrm[flip], axis=1, keepdims=True)
    hit = np.zeros((n, 20), np.float32)
    hit[:, 0:3], hit[:, 3:6], hit[:, 6:9], hit[:, 9] = nrm, ng, tan, hand
    hit[:, 10:13] = wi
    hit[:, 13:15] = rng.uniform(size=(n, 2))
    hit[:, 15:19] = 1.0
    hit[:, 19] = rng.integers(0, num_materials, n)
    rnd = rng.uniform(size=(n, 4)).astype(np.float32)
    return hit, wo.astype(np.float32), rnd


def random_rays(scene_vertices, n, seed=2, tfar=1e5):
    rng = np.random.default_rng(seed)
    p = scene_vertices[:, 0:3]
    lo, hi = p.min(0), p.max(0)
    org = rng.uniform(lo, hi, size=(n, 3))
    d = unit(rng, n)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3:6], rays[:, 6] = org, d, tfar
    return rays


def camera_rays_ref(ref, cam, width, height, n, seed=3):
    rng = np.random.default_rng(seed)
    xy = np.stack([rng.integers(0, width, n), rng.integers(0, height, n)], 1).astype(np.int32)
    r2 = rng.uniform(size=(n, 2)).astype(np.float32)
    return xy, r2


def load_golden():
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_small.npz")
    return dict(np.load(path))


def close_mask(a, b, rtol, atol):
    """Element-wise |a-b| <= atol + rtol|b|, treating equal infinities and NaN pairs as equal."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    with np.errstate(invalid="ignore"):
        near = np.abs(a - b) <= atol + rtol * np.abs(b)
    return same | near


def camera_of(scene):
    """PathtracingCamera of a synth.Scene's camera."""
    from dspbr.viewport import PathtracingCamera
    return PathtracingCamera(scene.camera.matrix_world, scene.camera.fov, scene.camera.near)
