"""ORACLE TEST INFRASTRUCTURE — not part of the product.

numpy restatement (float32, one rounding per operation) of the reference's
display passes: tonemap.frag (packages/lib/shader/tonemap.frag:20-94) and
fxaa.frag (:22-64) over RGBA32F images sampled NEAREST + CLAMP_TO_EDGE
(packages/lib/gl_utils.ts:22-30), and the 8-bit canvas conversion.  Checked
against the golden vectors the reference's own shaders produce
(tests/test_oracle_golden.py).
"""
import numpy as np

F = np.float32


def _gmax(x, y):  # GLSL max(x, y) = x < y ? y : x
    return np.where(x < y, y, x).astype(F)


def _gmin(x, y):  # GLSL min(x, y) = y < x ? y : x
    return np.where(y < x, y, x).astype(F)


def _sat(x):
    return _gmin(_gmax(x, F(0)), F(1))


def _u2(x):
    num = x * (F(0.15) * x + F(0.10) * F(0.50)) + F(0.20) * F(0.02)
    den = x * (F(0.15) * x + F(0.50)) + F(0.20) * F(0.30)
    return _gmax(num / den - F(0.02) / F(0.30), F(0))


_ACES_IN = np.array([[0.59719, 0.07600, 0.02840], [0.35458, 0.90834, 0.13383], [0.04823, 0.01566, 0.83777]], F)
_ACES_OUT = np.array([[1.60475, -0.10208, -0.00327], [-0.53108, 1.10813, -0.07276], [-0.07367, -0.00605, 1.07602]], F)


def _matmul(cols, v):  # mat3 (columns) * vec3, summed column by column
    return (cols[0] * v[..., 0:1] + cols[1] * v[..., 1:2]) + cols[2] * v[..., 2:3]


def tonemap(rgba, exposure, gamma, mode):
    """tonemap.frag main() per pixel; mode = renderer tonemappingModes index."""
    img = np.asarray(rgba, F)
    c = img[..., :3].copy()
    e = F(exposure)
    if mode == 0:
        c = e * c
    elif mode == 1:
        c = c * e
        c = _sat(c / (F(1) + c))
    elif mode == 2:
        c = c * e
        c = _gmax(F(0), c - F(0.004))
        c = np.power((c * (F(6.2) * c + F(0.5))) / (c * (F(6.2) * c + F(1.7)) + F(0.06)), F(2.2)).astype(F)
    elif mode == 3:
        c = c * (e / F(0.6))
        c = _matmul(_ACES_IN, c)
        a = c * (c + F(0.0245786)) - F(0.000090537)
        b = c * (F(0.983729) * c + F(0.4329510)) + F(0.238081)
        c = _matmul(_ACES_OUT, a / b)
        c = _sat(c)
    elif mode == 4:
        c = c * e
        c = _sat(_u2(c) / _u2(np.ones(3, F)))
    if gamma:
        c = np.power(c, F(1.0) / F(2.2)).astype(F)
    out = img.copy()
    out[..., :3] = c
    return out


def _tex(img, u, v):
    h, w = img.shape[:2]
    i = np.clip(np.floor(u * F(w)).astype(np.int64), 0, w - 1)
    j = np.clip(np.floor(v * F(h)).astype(np.int64), 0, h - 1)
    return img[j, i]


def fxaa(rgba):
    """fxaa.frag main() at every fragment centre."""
    img = np.asarray(rgba, F)
    h, w = img.shape[:2]
    inv = (F(1) / F(w), F(1) / F(h))
    y, x = np.mgrid[0:h, 0:w]
    fx, fy = x.astype(F) + F(0.5), y.astype(F) + F(0.5)
    t = lambda dx, dy: _tex(img, (fx + F(dx)) * inv[0], (fy + F(dy)) * inv[1])
    nw, ne, sw, se = t(-1, -1)[..., :3], t(1, -1)[..., :3], t(-1, 1)[..., :3], t(1, 1)[..., :3]
    cu, cv = fx * inv[0], fy * inv[1]
    tc = _tex(img, cu, cv)
    luma = np.array([0.299, 0.587, 0.114], F)
    dot = lambda a: (a[..., 0] * luma[0] + a[..., 1] * luma[1]) + a[..., 2] * luma[2]
    lnw, lne, lsw, lse, lm = dot(nw), dot(ne), dot(sw), dot(se), dot(tc[..., :3])
    lmin = _gmin(lm, _gmin(_gmin(lnw, lne), _gmin(lsw, lse)))
    lmax = _gmax(lm, _gmax(_gmax(lnw, lne), _gmax(lsw, lse)))
    dx = -((lnw + lne) - (lsw + lse))
    dy = (lnw + lsw) - (lne + lse)
    red = _gmax((((lnw + lne) + lsw) + lse) * (F(0.25) * (F(1) / F(8))), F(1) / F(128))
    rcp = F(1) / (_gmin(np.abs(dx), np.abs(dy)) + red)
    dx = _gmin(F(8), _gmax(F(-8), dx * rcp)) * inv[0]
    dy = _gmin(F(8), _gmax(F(-8), dy * rcp)) * inv[1]
    k1, k2 = F(1) / F(3) - F(0.5), F(2) / F(3) - F(0.5)
    s = lambda k: _tex(img, cu + dx * F(k), cv + dy * F(k))[..., :3]
    a = F(0.5) * (s(k1) + s(k2))
    b = a * F(0.5) + F(0.25) * (s(-0.5) + s(0.5))
    lb = dot(b)
    out = np.empty_like(img)
    use_a = (lb < lmin) | (lb > lmax)
    out[..., :3] = np.where(use_a[..., None], a, b)
    out[..., 3] = tc[..., 3]
    return out


def canvas8(rgba):
    """8-bit UNORM conversion of the canvas: round(clamp(c, 0, 1) * 255)."""
    return np.rint(np.clip(np.asarray(rgba, F), 0, 1) * F(255)).astype(np.uint8)
