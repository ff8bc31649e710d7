"""The spectral colour model on the host: RGB -> spectrum lifts, blackbody, sensor constants.

Host mirror of the reference's spectral machinery
(src/components/color/spectral/README.md; lookup.glsl / lookup.ts; spectra/blackbody):

* the bounded Jakob-Hanika lift (Jakob & Hanika, "A Low-Dimensional Function Space for
  Efficient Spectral Upsampling", 2019): rho(lambda) = clamp(0.5 + 0.5 p / sqrt(1 + p^2), 0, 1)
  with p = (a t + b) t + c and t = (lambda - 360) / 470;
* (a, b, c) by trilinear interpolation in the shipped 3 x 64^3 coefficient atlas: the largest
  RGB channel picks one of three tables (first channel wins ties), the other two divided by
  it are the horizontal coordinates, the maximum itself is located among 64 nonuniform
  nodes by six bisection steps (lookup.glsl:15-36, lookup.ts);
* reflectances (albedo, F0, tint) use the lift directly, coefficients (sigma_a, sigma_s) use
  scale = 2 max(rgb) and scale * rho(rgb / scale), emission additionally multiplies the D65
  curve (lookup.glsl:38-59); exact greys bypass the table;
* Planck emission relative to 550 nm with a CPU normalization to unit CIE Y
  (spectra/blackbody/blackbody.ts, blackbody.glsl:4-10).

Scene colours are constant, so the table lookup runs here, once per scene; the device
evaluates only the per-lane sigmoid polynomial of each lifted colour (``ptr_spectrum``).
The lookup arithmetic is float32 in the GLSL operation order (texelFetch + mix).

Data: the reference ships the model as two float32 assets, ``coefficients.bin`` (the atlas,
12.6 MB) and ``curves.bin`` (CIE 1931 x, y, z and D65 at 5 nm from 360 nm, and the 64
intensity nodes).  ``SpectralModel.from_assets(dir)`` loads them; ``SpectralModel.bundled()``
loads this package's subset (``data/jh_cie1931_d65_subset.npz``: the curves, the nodes and
the atlas nodes of the colours the package's workloads and tests use), made from the assets
by ``data/make_spectral_subset.py``.  A lookup that needs a node outside the loaded data
raises, naming the missing asset — like the reference's failed initialization by name.
"""
import math
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SUBSET = os.path.join(HERE, "data", "jh_cie1931_d65_subset.npz")
RES = 64
MODEL_VERSION = "jh-cie1931-d65-v1"   # the shipped colour model (color/spectral/data.ts:3)
LAMBDA_MIN, LAMBDA_MAX, STEP = 360.0, 830.0, 5.0
PLANCK_Q = 14387768.775039338      # h c / k in nm K (blackbody.glsl:5)

f32 = np.float32


def _mix(a, b, t):
    """GLSL mix in float32: a * (1 - t) + b * t."""
    a, b, t = f32(a), f32(b), f32(t)
    return f32(f32(a * f32(f32(1.0) - t)) + f32(b * t))


class MissingSpectralData(RuntimeError):
    pass


class SpectralModel:
    def __init__(self, curves, z_nodes, nodes, xyz_to_rgb=None):
        self.curves = np.ascontiguousarray(curves, dtype=np.float32).reshape(-1, 4)     # 95 x 4
        self.z_nodes = np.ascontiguousarray(z_nodes, dtype=np.float32).reshape(-1)     # 64
        self._nodes = nodes     # full atlas array (3, 64, 64, 64, 3) or dict flat-index -> (a, b, c)
        self.cie_y_integral = self._y_integral()
        # the model's own matrix when given (the reference's data.ts); else derived here
        self.xyz_to_rgb = np.asarray(xyz_to_rgb, np.float64) if xyz_to_rgb is not None else self._xyz_to_rgb()

    # ---- loading -----------------------------------------------------------------------
    @classmethod
    def from_assets(cls, data_dir):
        """The reference's shipped assets (coefficients.bin, curves.bin: RGBA float32 rows)."""
        cpath, kpath = os.path.join(data_dir, "curves.bin"), os.path.join(data_dir, "coefficients.bin")
        for p, size in ((cpath, 128 * 2 * 16), (kpath, 2048 * 384 * 16)):
            if not os.path.exists(p) or os.path.getsize(p) != size:
                raise MissingSpectralData(f"spectral asset missing or corrupt: {p}")
        cur = np.fromfile(cpath, dtype="<f4").reshape(2, 128, 4)
        atlas = np.fromfile(kpath, dtype="<f4").reshape(3, RES, RES, RES, 4)[..., :3]
        m = None
        ts = os.path.join(os.path.dirname(os.path.abspath(data_dir)), "data.ts")
        if os.path.exists(ts):   # the model's XYZ -> sRGB matrix, stored beside the assets
            import re
            block = re.search(r'"xyzToRGB":\s*\[(.*?)\]\s*\]', open(ts).read(), re.S)
            if block:
                m = np.array([float(v) for v in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", block.group(1))]).reshape(3, 3)
        return cls(cur[0, :95], cur[1, :RES, 0], atlas, m)

    @classmethod
    def bundled(cls):
        if not os.path.exists(SUBSET):
            raise MissingSpectralData(f"spectral asset missing: {SUBSET}")
        d = np.load(SUBSET)
        nodes = {int(k): tuple(v) for k, v in zip(d["node_index"], d["node_coef"])}
        return cls(d["curves"], d["z_nodes"], nodes, d["xyz_to_rgb"])

    def _node(self, channel, x, y, z):
        if isinstance(self._nodes, dict):
            idx = ((channel * RES + z) * RES + y) * RES + x
            if idx not in self._nodes:
                raise MissingSpectralData(f"spectral asset coefficients.bin: node {idx} is not in the loaded subset")
            return np.array(self._nodes[idx], np.float32)
        return self._nodes[channel, z, y, x].astype(np.float32)

    # ---- sensor constants (derived from the curves) ------------------------------------
    def _y_integral(self):
        """int ybar d lambda of the piecewise-linear 5 nm curve (trapezoid rule)."""
        y = self.curves[:, 1].astype(np.float64)
        return float(STEP * (y.sum() - 0.5 * (y[0] + y[-1])))

    def _xyz_to_rgb(self):
        """XYZ -> linear sRGB for the white point of these curves: the sRGB primaries
        (0.64, 0.33), (0.30, 0.60), (0.15, 0.06) and the D65 white integrated from the
        tabulated D65 and CMFs (unit Y)."""
        c = self.curves.astype(np.float64)
        xyz = STEP * (c[:, :3] * c[:, 3:4]).sum(axis=0) - 0.5 * STEP * (c[0, :3] * c[0, 3] + c[-1, :3] * c[-1, 3])
        white = xyz / xyz[1]
        prim = np.array([[0.64, 0.33], [0.30, 0.60], [0.15, 0.06]])
        P = np.stack([prim[:, 0] / prim[:, 1], np.ones(3), (1 - prim[:, 0] - prim[:, 1]) / prim[:, 1]])
        S = np.linalg.solve(P, white)
        return np.linalg.inv(P * S[None, :])

    # ---- the lifts ------------------------------------------------------------------------
    def coefficients(self, rgb):
        """(a, b, c) of the bounded lift of a non-grey rgb (lookup.glsl:15-36), float32."""
        r = [f32(v) for v in rgb]
        ch = 0 if (r[0] >= r[1] and r[0] >= r[2]) else (1 if r[1] >= r[2] else 2)
        z = r[ch]
        x = f32(f32(r[(ch + 1) % 3] / z) * f32(63.0))
        y = f32(f32(r[(ch + 2) % 3] / z) * f32(63.0))
        ix, iy = min(int(x), 62), min(int(y), 62)
        fx, fy = f32(x - f32(ix)), f32(y - f32(iy))
        lo, hi = 0, 63
        for _ in range(6):
            mid = (lo + hi) // 2
            if self.z_nodes[mid] <= z:
                lo = mid
            else:
                hi = mid
        z0, z1 = self.z_nodes[lo], self.z_nodes[lo + 1]
        fz = f32(f32(z - z0) / f32(z1 - z0))

        def plane(k):
            n00, n10 = self._node(ch, ix, iy, k), self._node(ch, ix + 1, iy, k)
            n01, n11 = self._node(ch, ix, iy + 1, k), self._node(ch, ix + 1, iy + 1, k)
            return [_mix(_mix(n00[c], n10[c], fx), _mix(n01[c], n11[c], fx), fy) for c in range(3)]
        a, b = plane(lo), plane(lo + 1)
        return [float(_mix(a[c], b[c], fz)) for c in range(3)]

    def nodes_of(self, rgb):
        """Flat atlas indices the lookup of rgb reads (for making data subsets)."""
        r = [f32(v) for v in rgb]
        if r[0] == r[1] == r[2]:
            return []
        ch = 0 if (r[0] >= r[1] and r[0] >= r[2]) else (1 if r[1] >= r[2] else 2)
        z = r[ch]
        x = f32(f32(r[(ch + 1) % 3] / z) * f32(63.0))
        y = f32(f32(r[(ch + 2) % 3] / z) * f32(63.0))
        ix, iy = min(int(x), 62), min(int(y), 62)
        lo, hi = 0, 63
        for _ in range(6):
            mid = (lo + hi) // 2
            if self.z_nodes[mid] <= z:
                lo = mid
            else:
                hi = mid
        return [((ch * RES + k) * RES + yy) * RES + xx for k in (lo, lo + 1) for yy in (iy, iy + 1) for xx in (ix, ix + 1)]

    @staticmethod
    def _spec(kind, c=(0.0, 0.0, 0.0), scale=1.0, d65=0):
        s = abi.Spectrum()
        s.kind = kind
        s.c = (abi.C.c_float * 3)(*c)
        s.scale = float(f32(scale))
        s.d65 = d65
        return s

    def reflectance(self, rgb):
        """color_lift_reflectance: the bounded lift (exact greys bypass the table)."""
        r = [float(f32(v)) for v in rgb]
        if r[0] == r[1] == r[2]:
            return self._spec(abi.SPEC_GREY, scale=r[0])
        return self._spec(abi.SPEC_LIFTED, c=self.coefficients(r), scale=1.0)

    def coefficient(self, rgb, d65=0):
        """color_lift_coefficient: scale = 2 max(rgb), scale * rho(rgb / scale)."""
        r = [f32(v) for v in rgb]
        scale = f32(f32(2.0) * max(r[0], max(r[1], r[2])))
        if scale == 0.0:
            return self._spec(abi.SPEC_GREY, scale=0.0, d65=d65)
        q = [f32(v / scale) for v in r]
        if q[0] == q[1] == q[2]:
            return self._spec(abi.SPEC_GREY, scale=float(f32(scale * q[0])), d65=d65)
        return self._spec(abi.SPEC_LIFTED, c=self.coefficients(q), scale=float(scale), d65=d65)

    def emission(self, rgb):
        """color_lift_emission: the coefficient lift times the D65 curve."""
        return self.coefficient(rgb, d65=1)

    def blackbody(self, kelvin, scale=1.0):
        """Planck radiance relative to 550 nm, normalized to unit reference CIE Y
        (blackbody.ts blackbodyColor: Simpson's rule on 0.5 nm steps in each 5 nm CMF
        interval), times scale."""
        c2 = 6.62607015e-34 * 299792458 / 1.380649e-23 * 1e9
        def shape(lam):
            return (550.0 / lam) ** 5 * math.expm1(c2 / (550.0 * kelvin)) / math.expm1(c2 / (lam * kelvin))
        cur = self.curves.astype(np.float64)
        y = 0.0
        for i in range(len(cur) - 1):
            for s in range(11):
                f = s / 10.0
                lam = LAMBDA_MIN + STEP * (i + f)
                w = 0.5 / 3.0 * (1 if s in (0, 10) else (4 if s % 2 else 2))
                y += w * shape(lam) / self.cie_y_integral * (cur[i, 1] * (1 - f) + cur[i + 1, 1] * f)
        return self._spec(abi.SPEC_BLACKBODY, c=(float(kelvin), 1.0 / y, 0.0), scale=scale)

    # ---- host evaluation (tests, quadrature witnesses) --------------------------------
    def curves_at(self, lam):
        lam = np.asarray(lam, np.float64)
        x = (lam - LAMBDA_MIN) / STEP
        i = np.minimum(np.floor(x).astype(int), 93)
        f = (x - i)[..., None]
        return self.curves[i].astype(np.float64) * (1 - f) + self.curves[i + 1].astype(np.float64) * f

    def eval(self, spec, lam):
        """float64 evaluation of a ptr_spectrum at wavelengths lam (for quadrature)."""
        lam = np.asarray(lam, np.float64)
        if spec.kind == abi.SPEC_GREY:
            v = np.full_like(lam, spec.scale)
        elif spec.kind == abi.SPEC_LIFTED:
            t = (lam - 360.0) / 470.0
            p = (spec.c[0] * t + spec.c[1]) * t + spec.c[2]
            v = spec.scale * np.clip(0.5 + 0.5 * p / np.sqrt(1 + p * p), 0.0, 1.0)
        else:
            q = PLANCK_Q / spec.c[0]
            r = 550.0 / lam
            v = spec.scale * spec.c[1] * np.expm1(q / 550.0) * r ** 5 / np.expm1(q / lam)
        if spec.d65:
            v = v * self.curves_at(lam)[..., 3]
        return v

    def sensor(self, lam):
        """sensor_response: XYZ -> linear sRGB of the CMFs at lam, over int ybar (cie1931.glsl:3-5)."""
        return (self.curves_at(lam)[..., :3] @ self.xyz_to_rgb.T) / self.cie_y_integral

    def spectral_desc(self, materials, lights, env):
        """The ptr_spectral_desc tables (host arrays kept on the returned object)."""
        return SpectralTables(self, materials, lights, env)


class SpectralTables:
    """Host-owned arrays of a ptr_spectral_desc."""

    def __init__(self, model, materials, lights, env):
        self.model = model
        self.materials = (abi.SpectralMaterial * max(1, len(materials)))(*materials)
        self.n_materials = len(materials)
        self.lights = (abi.Spectrum * max(1, len(lights)))(*lights)
        self.n_lights = len(lights)
        self.env = env
        self.curves = np.ascontiguousarray(model.curves, np.float32)

    def desc(self):
        d = abi.SpectralDesc()
        d.materials = self.materials
        d.lights = self.lights
        d.env = self.env
        d.curves = self.curves.ctypes.data_as(abi.C.POINTER(abi.C.c_float))
        d.xyz_to_rgb = (abi.C.c_float * 9)(*[float(v) for v in self.model.xyz_to_rgb.reshape(-1)])
        d.cie_y_integral = self.model.cie_y_integral
        return d


def wavelength_sample(u, kind="visible", lo=LAMBDA_MIN, hi=LAMBDA_MAX):
    """wavelengths_sample (spectral.glsl:1-10; visible.glsl / uniform.glsl) in float64:
    four cyclic quarter offsets of u in CDF space; returns (lambda[4], pdf[4])."""
    us = np.mod(u + 0.25 * np.arange(4), 1.0)
    if kind == "uniform":
        return lo + (hi - lo) * us, np.full(4, 1.0 / (hi - lo))
    a, b = math.tanh(0.0072 * (lo - 538.0)), math.tanh(0.0072 * (hi - 538.0))
    lam = 538.0 + np.arctanh(a * (1 - us) + b * us) / 0.0072
    c = np.cosh(0.0072 * (lam - 538.0))
    return lam, 0.0072 / ((b - a) * c * c)


def wavelength_density(lam, kind="visible", lo=LAMBDA_MIN, hi=LAMBDA_MAX):
    lam = np.asarray(lam, np.float64)
    if kind == "uniform":
        return np.full_like(lam, 1.0 / (hi - lo))
    a, b = math.tanh(0.0072 * (lo - 538.0)), math.tanh(0.0072 * (hi - 538.0))
    c = np.cosh(0.0072 * (lam - 538.0))
    return 0.0072 / ((b - a) * c * c)


def _blackbody_rgb(self, kelvin, scale=1.0):
    """blackbodyRGB (spectra/blackbody/blackbody.ts): the unit-Y Planck colour in linear
    sRGB times scale (RGB programs use it as the emission's stand-in)."""
    lam = np.linspace(LAMBDA_MIN, LAMBDA_MAX, 4701)
    spec = self.blackbody(kelvin, scale)
    v = self.eval(spec, lam)
    xyz = np.trapezoid(v[:, None] * self.curves_at(lam)[:, :3], lam, axis=0) / self.cie_y_integral
    return [float(x) for x in self.xyz_to_rgb @ xyz]


SpectralModel.blackbody_rgb = _blackbody_rgb
