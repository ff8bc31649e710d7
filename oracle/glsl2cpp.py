"""Translate one of the reference's generated GLSL fragment programs into C++20.

Test infrastructure for the oracle only.  The output compiles against
``oracle/glsl_compat.hpp`` and is linked into ``oracle/_ref/<case>.so``; it is the
reference's own transport program (``accumulation.ts:14-51`` main() and everything it
links) executed on the host.

The rewrite is purely lexical and deliberately small:
  * ``#version`` / ``precision`` lines are dropped; ``main`` becomes ``glsl_main``;
  * floating literals get an ``f`` suffix, so arithmetic stays binary32;
  * ``out T x`` / ``inout T x`` parameters become ``T& x``; ``in`` is dropped;
  * multi-letter swizzles (``.xyz``) become accessor calls (``.xyz()``);
  * file-scope variables (the RNG state ``rng_base``/``rng_dim``, ``fragColor``) become
    ``thread_local`` so pixels can run on several host threads;
  * ``uniform`` declarations become plain globals plus a name -> address table that
    the harness uses to bind values (the role of ``UniformBinding``,
    ``src/compiler/types.ts:793-812``, and ``RenderExecutor.executePass``).
"""
import re
import sys

_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
_SWIZZLE = re.compile(r"\.([xyzw]{2,4}|[rgba]{2,4})\b(?!\s*\()")
_PARAM_QUAL = re.compile(r"\b(inout|out)\s+(\w+)\s+(\w+)")
_IN_QUAL = re.compile(r"([(,]\s*)(?:const\s+)?in\s+(\w+\s+\w+)")
_UNIFORM = re.compile(r"^uniform\s+(\w+)\s+(\w+)\s*;")
_GLOBAL_VAR = re.compile(r"^(uint|int|float|bool|vec[234]|ivec[234]|uvec[234])\s+(\w+)\s*;")

_RANDOM_CALL = re.compile(r"\b(random2?)\(\)")

_UNIFORM_KIND = {
    "float": (0, 1), "vec2": (0, 2), "vec3": (0, 3), "vec4": (0, 4),
    "int": (1, 1), "ivec2": (1, 2), "ivec3": (1, 3), "ivec4": (1, 4),
    "uint": (2, 1), "bool": (3, 1),
    "sampler2D": (4, 0), "usampler2D": (5, 0),
}


def _strip_comment(line):
    i = line.find("//")
    return (line[:i], line[i:]) if i >= 0 else (line, "")


def _hoist_random(code):
    """GLSL evaluates call arguments left to right (GLSL ES 3.00 §6.1.1); C++ leaves the
    order unspecified.  A statement with two or more RNG draws (``vec2(random(),
    random())``, ``f(..., random(), random2())``) is rewritten to draw into temporaries
    in textual order first, so the dimension index sequence is the reference's."""
    calls = list(_RANDOM_CALL.finditer(code))
    if len(calls) < 2 or not code.rstrip().endswith(";"):
        return code
    indent = code[: len(code) - len(code.lstrip())]
    decls = []
    out = []
    last = 0
    for k, m in enumerate(calls):
        ty = "vec2" if m.group(1) == "random2" else "float"
        decls.append(f"{ty} _rng_h{k} = {m.group(1)}();")
        out.append(code[last:m.start()])
        out.append(f"_rng_h{k}")
        last = m.end()
    out.append(code[last:])
    stmt = "".join(out).strip()
    if stmt.startswith("return") or not re.match(r"^[A-Za-z_][\w<>]*\s+[A-Za-z_]\w*\s*=", stmt):
        return indent + "{ " + " ".join(decls) + " " + stmt + " }"
    # a declaration: keep the declared name visible after the statement
    return indent + " ".join(decls) + " " + stmt


def translate(src: str, ns: str):
    out = []
    uniforms = []
    depth = 0
    in_block_comment = False
    for raw in src.split("\n"):
        code, comment = _strip_comment(raw)
        if in_block_comment:
            if "*/" in code:
                in_block_comment = False
            out.append("// " + raw)
            continue
        if code.strip().startswith("/*") and "*/" not in code:
            in_block_comment = True
            out.append("// " + raw)
            continue
        s = code.strip()
        if s.startswith("#version") or s.startswith("precision "):
            out.append("// " + raw)
            continue
        if depth == 0:
            m = _UNIFORM.match(s)
            if m:
                uniforms.append((m.group(1), m.group(2)))
                out.append(f"{m.group(1)} {m.group(2)};")
                continue
            if s == "out vec4 fragColor;":
                out.append("thread_local vec4 fragColor;")
                continue
            if s == "out vec4 fragMoment;":
                out.append("thread_local vec4 fragMoment;")
                continue
            if _GLOBAL_VAR.match(s):
                code = "thread_local " + code
        if not s.startswith("#"):
            code = _FLOAT_LIT.sub(lambda m: m.group(1) + "f", code)
        else:
            # #define NAME 1.0  -> keep the define, suffix its floating value
            code = _FLOAT_LIT.sub(lambda m: m.group(1) + "f", code)
        code = _SWIZZLE.sub(lambda m: "." + m.group(1) + "()", code)
        code = _PARAM_QUAL.sub(lambda m: f"{m.group(2)}& {m.group(3)}", code)
        code = _IN_QUAL.sub(lambda m: m.group(1) + m.group(2), code)
        code = re.sub(r"\bnot\s*\(", "not_(", code)
        code = _hoist_random(code)
        code = re.sub(r"\bvoid\s+main\s*\(", "void glsl_main(", code)
        depth += code.count("{") - code.count("}")
        out.append(code + comment)
    body = "\n".join(out)

    table = []
    for ty, name in uniforms:
        kind, n = _UNIFORM_KIND[ty]
        table.append(f'    {{"{name}", {kind}, {n}, (void*)&{name}}},')
    has_stats = "Radiance transport_trace(Ray ray)" in src

    cpp = f"""// Generated by oracle/glsl2cpp.py from the reference's snapshot program.  Do not edit.
#include "glsl_compat.hpp"
#include <cstdio>
#include <cstring>
namespace glsl {{ namespace {ns} {{
thread_local vec4 gl_FragCoord;
{body}

struct UniformSlot {{ const char* name; int kind; int n; void* ptr; }};
static UniformSlot kUniforms[] = {{
{chr(10).join(table)}
    {{nullptr, 0, 0, nullptr}}
}};
}} }}  // namespace glsl::{ns}

using namespace glsl;
using namespace glsl::{ns};

// Bind a uniform by name (floats for float/int/uint/bool kinds).  Returns 0 on success.
extern "C" int ref_set_uniform(const char* name, const float* v, int n) {{
    for (UniformSlot* u = kUniforms; u->name; ++u) {{
        if (std::strcmp(u->name, name) != 0) continue;
        if (n != u->n) return -2;
        for (int i = 0; i < n; ++i) {{
            if (u->kind == 0) ((float*)u->ptr)[i] = v[i];
            else if (u->kind == 1) ((int*)u->ptr)[i] = (int)v[i];
            else if (u->kind == 2) ((unsigned*)u->ptr)[i] = (unsigned)v[i];
            else if (u->kind == 3) ((bool*)u->ptr)[i] = v[i] != 0.0f;
        }}
        return 0;
    }}
    return -1;
}}

extern "C" int ref_set_sampler(const char* name, const float* data, int w, int h) {{
    for (UniformSlot* u = kUniforms; u->name; ++u) {{
        if (std::strcmp(u->name, name) != 0) continue;
        if (u->kind == 4) {{ sampler2D* s = (sampler2D*)u->ptr; s->data = data; s->width = w; s->height = h; return 0; }}
        if (u->kind == 5) {{ usampler2D* s = (usampler2D*)u->ptr; s->data = (const unsigned*)data; s->width = w; s->height = h; return 0; }}
        return -2;
    }}
    return -1;
}}

extern "C" const char* ref_uniform_name(int i) {{
    int n = 0; for (UniformSlot* u = kUniforms; u->name; ++u) {{ if (n == i) return u->name; ++n; }}
    return nullptr;
}}

// The reference's own frame loop: for each sample, run main() over every pixel with
// u_sampleCount = s and u_previous bound to the previous frame, exactly the ping-pong
// of RenderExecutor (swap after each frame).  accum is W*H RGBA32F, row 0 = bottom.
extern "C" int ref_render_frames(int W, int H, int first_sample, int nframes, float* accum) {{
    float* prev = accum;
    float* cur = new float[(size_t)W * H * 4];
    for (int f = 0; f < nframes; ++f) {{
        float v = (float)(first_sample + f);
        ref_set_uniform("u_sampleCount", &v, 1);
        ref_set_sampler("u_previous", prev, W, H);
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < H; ++y) {{
            for (int x = 0; x < W; ++x) {{
                gl_FragCoord = vec4((float)x + 0.5f, (float)y + 0.5f, 0.5f, 1.0f);
                glsl_main();
                float* o = cur + 4 * ((size_t)y * W + x);
                o[0] = fragColor.x; o[1] = fragColor.y; o[2] = fragColor.z; o[3] = fragColor.w;
            }}
        }}
        std::memcpy(prev, cur, sizeof(float) * (size_t)W * H * 4);
    }}
    delete[] cur;
    return 0;
}}
"""
    if has_stats:
        cpp += f"""
// Per-sample statistics over the reference's own functions.  The body is main()'s
// camera-sample prologue (accumulation.ts:14-26 cameraSample): rng_init, pixel_sample,
// the lens draw, wavelengths_sample, camera_generateRay, transport_trace,
// color_to_pixel.  sum/sumsq are W*H*3 doubles (row 0 = bottom), accumulated in place.
extern "C" int ref_render_stats(int W, int H, int first_sample, int spp, double* sum, double* sumsq) {{
    #pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {{
        for (int x = 0; x < W; ++x) {{
            double* su = sum + 3 * ((size_t)y * W + x);
            double* sq = sumsq + 3 * ((size_t)y * W + x);
            for (int k = 0; k < spp; ++k) {{
                gl_FragCoord = vec4((float)x + 0.5f, (float)y + 0.5f, 0.5f, 1.0f);
                vec2 pixel = gl_FragCoord.xy() + u_pixelOffset;
                rng_init(uvec2(pixel), uint(first_sample + k), uint(u_resetSalt));
                vec2 film = pixel_sample(pixel, random2());
                vec2 xiLens = random2();
                (void)xiLens;
                WavelengthSample camera_sample = wavelengths_sample();
                Ray ray = camera_generateRay(film, xiLens, camera_sample.wl);
                Radiance L = transport_trace(ray);
                vec3 c = color_to_pixel(film, ray.direction, L, camera_sample);
                for (int ch = 0; ch < 3; ++ch) {{ su[ch] += (double)c[ch]; sq[ch] += (double)c[ch] * (double)c[ch]; }}
            }}
        }}
    }}
    return 0;
}}
"""
    return cpp


def main(argv):
    src = open(argv[1], encoding="utf-8").read()
    ns = argv[3]
    with open(argv[2], "w", encoding="utf-8") as f:
        f.write(translate(src, ns))


if __name__ == "__main__":
    main(sys.argv)
