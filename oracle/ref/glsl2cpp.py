#!/usr/bin/env python3
"""ORACLE TEST INFRASTRUCTURE — not part of the product.

Build-time recipe that turns the reference's own GLSL fragment shader
(packages/lib/shader/renderer.frag and the chunks it includes) into C++ that
compiles against glsl_shim.h.  The output is written ONLY to oracle/_ref/
(git-ignored); no reference source is committed to this repository.

The chunk order reproduces the `#include` order of renderer.frag:47-63 and the
chunk map of renderer.ts:1072-1094 (`pbr_kernel` = the webgl-full material
profile, `integrator` = integrator/misptdl.glsl).  Chunks that the reference
generates at run time from TypeScript (`buffer_accessor`, `texture_accessor`,
`material_block`, `mesh_constants`, `lights`) are supplied by the hand-written
C++ files in oracle/ref/chunks/.

Rewrites (all mechanical, checked by counting expected matches):
  * qualifiers in parameter lists: `const in T` -> `const T`, `in T` -> `T`,
    `out T x` / `inout T x` -> `T& x`, `inout int a[N]` -> `int* a`;
  * swizzles `.xyz .rgb .xy .yx .zw .rg` -> accessor calls, and the two
    swizzle assignments (material.glsl) -> setter calls;
  * float literals get an `f` suffix in the FP32 build;
  * GLSL evaluates call arguments left to right (GLSL ES 3.00 5.10); C++ does
    not, so the three call sites that pass several `rng_float()` arguments are
    rewritten into sequenced temporaries;
  * locals and `out` parameters are zero-initialised, as WebGL's shader
    translator does (GLSL itself leaves them undefined; this decides e.g. the
    `event_type` field that configure_gltf_material never writes);
  * `void main()` -> `void glsl_main()`; `float` -> `real`; the global RNG
    state becomes thread_local; `INFINITY` (a libm macro) is renamed.
"""
import argparse
import os
import re
import sys

SHADER_DIR = "packages/lib/shader"
CHUNKS = {
    "pbr_kernel": "generated/slang_materials/webgl-full/material_kernel.glsl",
    "structs": "structs.glsl",
    "rng": "rng.glsl",
    "constants": "constants.glsl",
    "utils": "utils.glsl",
    "material": "material.glsl",
    "bvh": "bvh.glsl",
    "pbr_material_adapter": "pbr_material_adapter.glsl",
    "lighting": "lighting.glsl",
    "integrator": "integrator/misptdl.glsl",
}
LOCAL_CHUNKS = ["buffer_accessor", "texture_accessor", "material_block", "mesh_constants", "lights"]
KEYWORDS = {"if", "for", "while", "switch", "return", "else"}


def expect(n, want, what):
    if n != want:
        raise SystemExit(f"glsl2cpp: expected {want} rewrite(s) of {what}, found {n}")


def rewrite_params(src):
    func_re = re.compile(r"\b([A-Za-z_]\w*)(\s+)([A-Za-z_]\w*)(\s*)\(([^(){};]*)\)(\s*\{)", re.S)

    def fix(m):
        ret, name = m.group(1), m.group(3)
        if ret in KEYWORDS or name in KEYWORDS:
            return m.group(0)
        params = m.group(5)
        params = re.sub(r"\bconst\s+in\b", "const", params)
        params = re.sub(r"\binout\s+(\w+)\s+(\w+)\s*\[\s*\w+\s*\]", r"\1* \2", params)
        outs = re.findall(r"\bout\s+(\w+)\s+(\w+)", params)
        params = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)", r"\1& \2", params)
        params = re.sub(r"\bin\s+", "", params)
        init = "".join(f" {n} = {t}{{}};" for t, n in outs)
        return f"{ret}{m.group(2)}{name}{m.group(4)}({params}){m.group(6)}{init}"

    return func_re.sub(fix, src)


BASE_TYPES = ["real", "float", "int", "uint", "bool", "vec2", "vec3", "vec4", "ivec2", "uvec2", "mat3", "mat4"]


def zero_init(src):
    """WebGL's shader translator zero-initialises locals and `out` parameters
    (GLSL leaves them undefined).  Emulate it: `T a, b;` -> `T a{}, b{};` and
    each `out` parameter is assigned `T{}` on function entry."""
    structs = re.findall(r"\bstruct\s+(\w+)", src)
    types = "(?:" + "|".join(BASE_TYPES + structs) + ")"
    decl = re.compile(r"^(\s*)(" + types + r")\s+(\w+(?:\s*\[\s*\w+\s*\])?(?:\s*,\s*\w+)*)\s*;", re.M)

    def fix_decl(m):
        if m.group(2) in ("return", "else"):
            return m.group(0)
        names = [n.strip() for n in m.group(3).split(",")]
        return m.group(1) + m.group(2) + " " + ", ".join(n + "{}" for n in names) + ";"

    return decl.sub(fix_decl, src)


def rewrite_swizzles(src):
    # swizzle assignments first (material.glsl:95 and :13)
    src, n1 = re.subn(r"([\w.]+)\.(xyz|rgb)\s*=\s*([^;=][^;]*);", r"\1.set_\2(\3);", src)
    src, n2 = re.subn(r"([\w.]+)\.(xyz|rgb)\s*\*=\s*([^;]*);", r"\1.mul_\2(\3);", src)
    expect(n1, 1, "swizzle assignment")
    expect(n2, 1, "swizzle multiply-assignment")
    src = re.sub(r"\.(xyz|rgb|xy|yx|zw|rg)\b(?!\s*\()", r".\1()", src)
    return src


FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def rewrite_literals(src, fp32):
    if not fp32:
        return src
    out = []
    for line in src.split("\n"):
        if line.lstrip().startswith("//"):
            out.append(line)
            continue
        out.append(FLOAT_LIT.sub(lambda m: m.group(1) + "f", line))
    return "\n".join(out)


def sequence_rng_args(src):
    # renderer.frag:106  vec3(rng_float(), rng_float(), rng_float())
    src, n = re.subn(
        r"rs\.wo = pbr_material_sample\(rs\.closure, rs\.wi,\s*vec3\(rng_float\(\), rng_float\(\), rng_float\(\)\),",
        "real u0_ = rng_float(); real u1_ = rng_float(); real u2_ = rng_float();\n"
        "    rs.wo = pbr_material_sample(rs.closure, rs.wi, vec3(u0_, u1_, u2_),",
        src)
    expect(n, 1, "pbr_material_sample rng arguments")
    # misptdl.glsl:72  eval_direct_light_contribution(rs, rng_float(), rng_float())
    src, n = re.subn(
        r"L \+= eval_direct_light_contribution\(rs, rng_float\(\), rng_float\(\)\) \* path_weight;",
        "{ real r0_ = rng_float(); real r1_ = rng_float();\n"
        "      L += eval_direct_light_contribution(rs, r0_, r1_) * path_weight; }",
        src)
    expect(n, 1, "eval_direct_light_contribution rng arguments")
    # renderer.frag:149  calcuateViewRay(rng_float(), rng_float())
    src, n = re.subn(
        r"bvh_ray r = calcuateViewRay\(rng_float\(\), rng_float\(\)\);",
        "real c0_ = rng_float(); real c1_ = rng_float();\n  bvh_ray r = calcuateViewRay(c0_, c1_);",
        src)
    expect(n, 1, "calcuateViewRay rng arguments")
    return src


def strip_frag_header(src):
    src = re.sub(r"#version[^\n]*\n", "", src)
    src = re.sub(r"precision\s+\w+\s+\w+\s*;", "", src)
    src, n = re.subn(r"layout\(std140\)\s*uniform\s+PathTracingUniformBlock\s*\{.*?\};", "", src, flags=re.S)
    expect(n, 1, "uniform block")
    src = re.sub(r"\buniform\s+\w+\s+\w+\s*;", "", src)
    src = re.sub(r"\bin\s+vec2\s+v_uv\s*;", "", src)
    src = re.sub(r"layout\(location\s*=\s*0\)\s*out\s+vec4\s+out_FragColor\s*;", "", src)
    return src


def translate(ref_root, chunk_dir, fp32):
    sd = os.path.join(ref_root, SHADER_DIR)
    with open(os.path.join(sd, "renderer.frag")) as f:
        frag = f.read()
    frag = strip_frag_header(frag)

    def include(m):
        name = m.group(1)
        if name in CHUNKS:
            with open(os.path.join(sd, CHUNKS[name])) as f:
                text = f.read()
            text = re.sub(r"precision\s+\w+\s+\w+\s*;", "", text)
            return f"\n// ---- chunk <{name}> from {CHUNKS[name]}\n{text}\n"
        if name in LOCAL_CHUNKS:
            with open(os.path.join(chunk_dir, name + ".inc")) as f:
                return f"\n// ---- chunk <{name}> (host restatement)\n{f.read()}\n"
        raise SystemExit(f"glsl2cpp: unknown chunk <{name}>")

    src = re.sub(r"#include\s*<(\w+)>", include, frag)
    src = sequence_rng_args(src)
    src, n = re.subn(r"^uvec2 rng_state;", "thread_local uvec2 rng_state;", src, flags=re.M)
    expect(n, 1, "rng_state global")
    src = zero_init(src)
    src = rewrite_params(src)
    src = rewrite_swizzles(src)
    src, n = re.subn(r"\bvoid\s+main\s*\(\s*\)", "void glsl_main()", src)
    expect(n, 1, "main")
    src = re.sub(r"\bINFINITY\b", "GLSL_INFINITY", src)
    # lighting.glsl:15 declares a local `isVisible` initialised by the function
    # of the same name; GLSL scopes the name after its initializer, C++ before.
    src, n = re.subn(r"bool isVisible = isVisible\(", "bool isVisible = glsl::isVisible(", src)
    expect(n, 1, "isVisible shadowing")
    # instrumentation for the CPU baseline: count traced rays (every closest-hit
    # and shadow query goes through intersectSceneTriangles_BVH, bvh.glsl:149)
    src, n = re.subn(r"(bool intersectSceneTriangles_BVH\([^)]*\)\s*\{)", r"\1 ++glsl_rays_traced;", src)
    expect(n, 1, "ray counter hook")
    src = re.sub(r"\bfloat\b", "real", src)
    src = rewrite_literals(src, fp32)
    return src


POST_SHADERS = {"tonemap": "tonemap.frag", "fxaa": "fxaa.frag"}


def translate_post(ref_root, fp32):
    """The display epilogue shaders (tonemap.frag, fxaa.frag), each in its own
    namespace.  Their uniforms become namespace globals the harness sets;
    `in v_uv` / `out` colour / gl_FragCoord are the harness's per-fragment
    built-ins.  The output variable is renamed to out_FragColor."""
    sd = os.path.join(ref_root, SHADER_DIR)
    parts = []
    for ns, fname in POST_SHADERS.items():
        with open(os.path.join(sd, fname)) as f:
            src = f.read()
        src = re.sub(r"#version[^\n]*\n", "", src)
        src = re.sub(r"precision\s+\w+\s+\w+\s*;", "", src)
        src = re.sub(r"\b(?:mediump|highp|lowp)\s+", "", src)
        src, n = re.subn(r"\buniform\s+", "", src)
        expect(n >= 2, True, f"uniforms of {fname}")
        src = re.sub(r"\bin\s+vec2\s+v_uv\s*;", "", src)
        src, n = re.subn(r"\bout\s+vec4\s+(\w+)\s*;", "", src)
        expect(n, 1, f"output of {fname}")
        src = re.sub(r"\bout_color\b", "out_FragColor", src)
        src = zero_init(src)
        src = rewrite_params(src)
        src = re.sub(r"\.(xyz|rgb|xy|yx|zw|rg)\b(?!\s*\()", r".\1()", src)
        src, n = re.subn(r"\bvoid\s+main\s*\(\s*\)", "void glsl_main()", src)
        expect(n, 1, f"main of {fname}")
        src = re.sub(r"\bfloat\b", "real", src)
        src = rewrite_literals(src, fp32)
        parts.append(f"namespace post_{ns} {{\n// ---- {fname}\n{src}\n}}  // namespace post_{ns}\n")
    return "\n".join(parts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference checkout")
    ap.add_argument("--chunks", required=True)
    ap.add_argument("--out", required=True)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--post", action="store_true", help="translate the display epilogue shaders instead")
    a = ap.parse_args()
    src = translate_post(a.ref, fp32=not a.fp64) if a.post else translate(a.ref, a.chunks, fp32=not a.fp64)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    with open(a.out, "w") as f:
        f.write("// GENERATED at build time from the reference shaders; not committed.\n")
        f.write(src)
    return 0


if __name__ == "__main__":
    sys.exit(main())
