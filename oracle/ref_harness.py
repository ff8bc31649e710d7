"""Drive the reference's own generated programs (compiled into ``oracle/_ref/*.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` and by the golden-fixture script,
never by the product.

Each ``oracle/_ref/<case>.so`` is one snapshot program translated by
``oracle/glsl2cpp.py``.  This module binds its uniforms exactly as the reference
computes them on the host and runs it:

* camera basis  -> ``src/components/camera/basis.ts:49-55`` (``cameraBasis``)
* ``u_tanFov = tan(fov/2)`` -> ``src/compiler/generate/features/camera.ts:62-65``
* ``u_aspect = w/h``       -> ``camera.ts:121-127``
* engine builtins (sampleCount, resetSalt, pixelOffset, imageSize)
  -> ``src/engine/Engine.ts:231-258``
* every other uniform takes its parameter's default from the renderer's
  ``parameters`` table (``UniformBinding.compute`` of a plain parameter).

WebGL uploads JS doubles as binary32, so every value is rounded to float32 here.
"""
import ctypes
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def camera_basis(position, target):
    """``cameraBasis`` (basis.ts:49-55), in float64 like the TypeScript."""
    def sub(a, b):
        return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]

    def cross(a, b):
        return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]

    def normalize(v):
        n = math.hypot(v[0], v[1], v[2])
        return [v[0] / n, v[1] / n, v[2] / n]

    forward = normalize(sub(target, position))
    up_ref = [0.0, 0.0, 1.0] if abs(forward[1]) > 0.999999 else [0.0, 1.0, 0.0]
    right = normalize(cross(forward, up_ref))
    up = cross(right, forward)
    return forward, right, up


def available():
    return os.path.exists(os.path.join(REF_DIR, "index.json"))


def cases():
    with open(os.path.join(REF_DIR, "index.json")) as f:
        return json.load(f)


class RefProgram:
    """One reference program; ``stats`` returns per-pixel mean and variance."""

    def __init__(self, case):
        idx = cases()
        if case not in idx or not idx[case].get("built"):
            raise FileNotFoundError(f"reference program {case!r} not built in {REF_DIR}")
        self.case = case
        self.meta = idx[case]
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, case + ".so"))
        self.lib.ref_set_uniform.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int]
        self.lib.ref_set_sampler.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        self.lib.ref_render_frames.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        if hasattr(self.lib, "ref_render_stats"):
            self.lib.ref_render_stats.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p] * 2
        self._keep = []

    def defaults(self):
        return {k: v.get("default") for k, v in self.meta.get("parameters", {}).items()}

    def set_uniform(self, name, values):
        vals = [float(np.float32(v)) for v in (values if isinstance(values, (list, tuple)) else [values])]
        arr = (ctypes.c_float * len(vals))(*vals)
        rc = self.lib.ref_set_uniform(name.encode(), arr, len(vals))
        if rc == -2:
            raise ValueError(f"{self.case}: uniform {name} given {len(vals)} values")
        return rc == 0

    def bind(self, width, height, salt=0, params=None):
        """Bind every uniform the program declares (sampleCount is set per frame)."""
        p = self.defaults()
        p.update(params or {})
        pos = p.get("camera.position") or [0, 0, 8]
        tgt = p.get("camera.target") or [0, 0, 0]
        fov = p.get("camera.fov", 0.8)
        fwd, right, up = camera_basis(pos, tgt)
        derived = {
            "u_cameraPosition": pos, "u_cameraForward": fwd, "u_cameraRight": right, "u_cameraUp": up,
            "u_imageSize": [width, height], "u_resolution": [width, height],
            "u_aspect": width / height if height else 1.0,
            "u_tanFov": math.tan(fov / 2.0), "u_resetSalt": salt, "u_pixelOffset": [0.0, 0.0],
        }
        for u in self.meta.get("uniforms", []):
            name = u["uniform"]
            if name in derived or name == "u_sampleCount":
                continue
            paths = u.get("parameters", [])
            if len(paths) == 1 and paths[0] in p and p[paths[0]] is not None:
                self.set_uniform(name, p[paths[0]])
            else:
                raise ValueError(f"{self.case}: no binding rule for uniform {name} ({paths})")
        for name, val in derived.items():
            self.set_uniform(name, val)

    def stats(self, width, height, spp, first_sample=0):
        """Per-pixel mean and unbiased variance of ``spp`` samples (rows bottom-up)."""
        s = np.zeros((height, width, 3), np.float64)
        q = np.zeros((height, width, 3), np.float64)
        self.lib.ref_render_stats(width, height, first_sample, spp, s.ctypes.data, q.ctypes.data)
        mean = s / spp
        var = np.maximum(q / spp - mean * mean, 0.0) * (spp / max(spp - 1, 1))
        return mean, var

    def frames(self, width, height, nframes, first_sample=0, accum=None):
        """The reference's own running-mean film after ``nframes`` frames (RGBA)."""
        if accum is None:
            accum = np.zeros((height, width, 4), np.float32)
        accum = np.ascontiguousarray(accum, np.float32)
        self.lib.ref_render_frames(width, height, first_sample, nframes, accum.ctypes.data)
        return accum
