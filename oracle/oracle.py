"""Python binding of the CPU restatement (``oracle/pt_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / reference arm of ``bench.py`` as the checker, never by the product.
It consumes the same packed scene (``include/ptx_rt.h`` layout) the CUDA engine uploads.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")
# the same restatement with its float transcendentals evaluated in double and rounded once
# (a second binary32 libm; see fm in pt_oracle.cpp)
LIB_WIDE = os.path.join(BUILD, "liboracle_wide.so")
SOURCES = [os.path.join(HERE, "pt_oracle.cpp")]


def build(force=False):
    """Compile the restatement with g++ (OpenMP, -O3, binary32 without FMA contraction),
    and its wide-transcendental twin."""
    os.makedirs(BUILD, exist_ok=True)
    header = os.path.join(HERE, "..", "include", "ptx_rt.h")
    newest = max(os.path.getmtime(p) for p in SOURCES + [header])
    for out, extra in ((LIB, []), (LIB_WIDE, ["-DORACLE_WIDE_MATH"])):
        if not force and os.path.exists(out) and os.path.getmtime(out) >= newest:
            continue
        cmd = ["g++", "-std=c++17", "-O3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", *extra,
               *SOURCES, "-o", out + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(out + ".tmp", out)
    return LIB


_libs = {}


def lib(variant=""):
    """The oracle library: "" (the host libm's float functions) or "wide"."""
    if variant not in _libs:
        path = LIB_WIDE if variant == "wide" else LIB
        if not os.path.exists(path):
            build()
        _lib = ctypes.CDLL(path)
        _libs[variant] = _lib
        _lib.oracle_render.restype = ctypes.c_int
        _lib.oracle_render.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_void_p] * 3 + [ctypes.c_void_p, ctypes.c_int]
        _lib.oracle_render_tile.restype = ctypes.c_int
        _lib.oracle_render_tile.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        _lib.oracle_session_create.restype = ctypes.c_void_p
        _lib.oracle_session_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_session_free.argtypes = [ctypes.c_void_p]
        _lib.oracle_session_render_tile.restype = ctypes.c_int
        _lib.oracle_session_render_tile.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        _lib.oracle_trace_closest.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_mesh_brute.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_rough_dielectric_eval_n.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float] + [ctypes.c_void_p] * 5
        _lib.oracle_rough_dielectric_sample_n.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float] + [ctypes.c_void_p] * 7
        _lib.oracle_field_eval.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        _lib.oracle_forward_tile.restype = ctypes.c_int
        _lib.oracle_forward_tile.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 2 + [ctypes.c_int]
    return _libs[variant]


def render(packed, renderer, width, height, spp, first_sample=0, salt=0, params=None,
           threads=0, keep_samples=False, pixel_offset=(0, 0), image_size=None, variant=""):
    """Render with the oracle.  Returns dict(mean, var, sum, sumsq, samples?, counts).
    ``pixel_offset`` / ``image_size``: the frame is a width x height tile at that offset of
    an image of that size (engine.pixelOffset / engine.imageSize).  ``variant``: "" or
    "wide" (the twin whose float transcendentals are evaluated in double)."""
    from pathtracerglsl_b200 import abi
    desc = packed.desc()
    fr = abi.Frame()
    fr.width, fr.height = width, height
    fr.first_sample, fr.spp = first_sample, spp
    fr.reset_salt = salt
    fr.pixel_offset = (ctypes.c_int32 * 2)(*pixel_offset)
    iw, ih = image_size or (width, height)
    fr.image_size = (ctypes.c_int32 * 2)(iw, ih)
    fr.camera = renderer.camera(params or {}, iw, ih)
    s = np.zeros((height, width, 3), np.float64)
    q = np.zeros((height, width, 3), np.float64)
    samples = np.zeros((spp, height, width, 3), np.float32) if keep_samples else None
    counts = (ctypes.c_uint64 * 2)()
    rc = lib(variant).oracle_render(ctypes.addressof(desc), ctypes.addressof(renderer.program), ctypes.addressof(fr),
                             s.ctypes.data, q.ctypes.data,
                             samples.ctypes.data if samples is not None else None,
                             ctypes.addressof(counts), threads)
    if rc != 0:
        raise RuntimeError(f"oracle_render failed: {rc}")
    mean = s / spp
    var = np.maximum(q / spp - mean * mean, 0.0) * (spp / max(spp - 1, 1))
    out = {"mean": mean, "var": var, "sum": s, "sumsq": q,
           "closest_queries": counts[0], "shadow_queries": counts[1]}
    if samples is not None:
        out["samples"] = samples
    return out


def forward(packed, renderer, width, height, spp, first_sample=0, salt=0, params=None, threads=0):
    """Forward-mode reference of the path-replay adjoint (float64 tangents along the
    oracle's own walk, same random numbers as a render with the same frame).  Returns
    dict(jac, mean): jac[y, x, c, PTR_GRAD_SLOTS * material + slot] = d I / d theta of the
    pixel's mean over the frame's samples, row 0 = bottom; mean = the image itself."""
    from pathtracerglsl_b200 import abi
    desc = packed.desc()
    fr = abi.Frame()
    fr.width, fr.height = width, height
    fr.first_sample, fr.spp = first_sample, spp
    fr.reset_salt = salt
    fr.camera = renderer.camera(params or {}, width, height)
    K = abi.GRAD_SLOTS * len(packed.materials)
    jac = np.zeros((height, width, 3, K), np.float64)
    s = np.zeros((height, width, 3), np.float64)
    rc = lib().oracle_forward_tile(ctypes.addressof(desc), ctypes.addressof(renderer.program), ctypes.addressof(fr),
                                   0, 0, width, height, jac.ctypes.data, s.ctypes.data, threads)
    if rc == -2:
        raise ValueError("forward mode covers the adjoint's model only: RGB, no equiangular NEE, grey media")
    if rc != 0:
        raise RuntimeError(f"oracle_forward_tile failed: {rc}")
    return {"jac": jac / spp, "mean": s / spp}


def field_eval(code, points):
    """The oracle's interpretation of a coefficient field program at points (n, 3)."""
    code = np.ascontiguousarray(code, np.uint32)
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    out = np.zeros(p.shape, np.float32)
    lib().oracle_field_eval(code.ctypes.data, 0, p.ctypes.data, len(p), out.ctypes.data)
    return out


def rough_dielectric_eval(alpha, n_i, n_t, wi, wo, tint=(1.0, 1.0, 1.0)):
    """The oracle's rough dielectric in its local frame (n = +z): f (n, 3) and pdf (n,) for
    direction arrays wi, wo (n, 3)."""
    wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
    wo = np.ascontiguousarray(np.broadcast_to(np.asarray(wo, np.float32), wi.shape))
    t = np.ascontiguousarray(tint, np.float32)
    f = np.zeros(wi.shape, np.float32)
    pdf = np.zeros(len(wi), np.float32)
    lib().oracle_rough_dielectric_eval_n(len(wi), alpha, n_i, n_t, t.ctypes.data, wi.ctypes.data, wo.ctypes.data,
                                         f.ctypes.data, pdf.ctypes.data)
    return f, pdf


def rough_dielectric_sample(alpha, n_i, n_t, wo, u, tint=(1.0, 1.0, 1.0)):
    """One sample per row of u (n, 3) = (uc, u0, u1): wi (n, 3), weight (n, 3), pdf, flags."""
    u = np.ascontiguousarray(u, np.float32).reshape(-1, 3)
    wo = np.ascontiguousarray(np.broadcast_to(np.asarray(wo, np.float32), u.shape))
    t = np.ascontiguousarray(tint, np.float32)
    wi = np.zeros(u.shape, np.float32)
    w = np.zeros(u.shape, np.float32)
    pdf = np.zeros(len(u), np.float32)
    flags = np.zeros(len(u), np.int32)
    lib().oracle_rough_dielectric_sample_n(len(u), alpha, n_i, n_t, t.ctypes.data, wo.ctypes.data, u.ctypes.data,
                                           wi.ctypes.data, w.ctypes.data, pdf.ctypes.data, flags.ctypes.data)
    return wi, w, pdf, flags


def render_tile(packed, renderer, width, height, tile, spp, first_sample=0, salt=0, params=None, threads=0):
    """Render the tile (x0, y0, tw, th) of a width x height image; returns (mean, counts)."""
    from pathtracerglsl_b200 import abi
    x0, y0, tw, th = tile
    desc = packed.desc()
    fr = abi.Frame()
    fr.width, fr.height = width, height
    fr.first_sample, fr.spp = first_sample, spp
    fr.reset_salt = salt
    fr.camera = renderer.camera(params or {}, width, height)
    s = np.zeros((th, tw, 3), np.float64)
    q = np.zeros((th, tw, 3), np.float64)
    counts = (ctypes.c_uint64 * 2)()
    rc = lib().oracle_render_tile(ctypes.addressof(desc), ctypes.addressof(renderer.program), ctypes.addressof(fr),
                                  x0, y0, tw, th, s.ctypes.data, q.ctypes.data, None, ctypes.addressof(counts), threads)
    if rc != 0:
        raise RuntimeError(f"oracle_render_tile failed: {rc}")
    return s / spp, (counts[0], counts[1])


class Session:
    """A scene prepared once (the oracle's mesh acceleration built), rendered many times."""

    def __init__(self, packed, renderer):
        self.packed, self.renderer = packed, renderer
        self._desc = packed.desc()
        self._h = lib().oracle_session_create(ctypes.addressof(self._desc), ctypes.addressof(renderer.program))

    def render_tile(self, width, height, tile, spp, first_sample=0, salt=0, params=None, threads=0):
        from pathtracerglsl_b200 import abi
        x0, y0, tw, th = tile
        fr = abi.Frame()
        fr.width, fr.height = width, height
        fr.first_sample, fr.spp = first_sample, spp
        fr.reset_salt = salt
        fr.camera = self.renderer.camera(params or {}, width, height)
        s = np.zeros((th, tw, 3), np.float64)
        q = np.zeros((th, tw, 3), np.float64)
        counts = (ctypes.c_uint64 * 2)()
        rc = lib().oracle_session_render_tile(self._h, ctypes.addressof(fr), x0, y0, tw, th, s.ctypes.data, q.ctypes.data,
                                              None, ctypes.addressof(counts), threads)
        if rc != 0:
            raise RuntimeError(f"oracle_session_render_tile failed: {rc}")
        return s / spp, (counts[0], counts[1])

    def close(self):
        if self._h:
            lib().oracle_session_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def trace_closest(packed, renderer, rays):
    """Nearest hit per ray (rays: n x 6 float32 origin, direction) -> (region, instance,
    prim, t); ties at equal t go to the lower region, instance and triangle index."""
    rays = np.ascontiguousarray(rays, np.float32)
    n = len(rays)
    region = np.zeros(n, np.int32)
    element = np.zeros(n, np.int32)
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    desc = packed.desc()
    lib().oracle_trace_closest(ctypes.addressof(desc), ctypes.addressof(renderer.program), rays.ctypes.data, n,
                               region.ctypes.data, element.ctypes.data, prim.ctypes.data, t.ctypes.data)
    return region, element, prim, t


def mesh_brute(packed, mesh_index, rays):
    """Brute-force nearest triangle of one packed mesh -> (prim, t)."""
    rays = np.ascontiguousarray(rays, np.float32)
    n = len(rays)
    prim = np.zeros(n, np.int32)
    t = np.zeros(n, np.float32)
    desc = packed.desc()
    lib().oracle_mesh_brute(ctypes.addressof(desc.meshes[mesh_index]), rays.ctypes.data, n, prim.ctypes.data, t.ctypes.data)
    return prim, t
