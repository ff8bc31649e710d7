"""Differentiable material parameters of a packed scene (the adjoint's parameter space).

No counterpart in the reference, which renders only.  Per material there are
``abi.GRAD_SLOTS`` parameters, laid out as the C ABI's PTR_GRAD_* slots:

* the model's colour r, g, b: Lambert albedo, GGX / mirror F0, dielectric transmittance;
* GGX alpha;
* dielectric IOR, the IOR of every region the material is attached to;
* for a grey homogeneous medium: sigma_t = sigma_a + sigma_s, the single-scattering albedo
  a = sigma_s / sigma_t, and the HG asymmetry g.

``param_table`` reads them, ``with_params`` writes a modified copy (regions included), and
``live_mask`` tells which slots a material's model uses.  ``CudaEngine.backward`` returns
gradients in the same (n_materials, GRAD_SLOTS) layout, and ``CudaEngine.update_params``
pushes an edited copy to the device.
"""
import copy

import numpy as np

from . import abi
from . import occupants


def _materials(packed):
    return (abi.Material * len(packed.materials)).from_buffer(packed.materials)


def _regions(packed):
    return (abi.Region * len(packed.regions)).from_buffer(packed.regions)


def _color_field(m):
    """The ptr_material field of a material's colour parameter (slots 0-2): its model's
    registry row names it (albedo where the model differentiates no colour)."""
    row = occupants.MATERIAL_BY_ID.get(m.model)
    return (row.grad_color if row is not None else None) or "albedo"


def _color(m):
    """The colour parameter of a material's model (slots 0-2)."""
    return getattr(m, _color_field(m))


def live_mask(packed):
    """(n_materials, GRAD_SLOTS) bool: the slots each material's model uses."""
    mats = _materials(packed)
    regs = _regions(packed)
    used = {r.material for r in regs}
    mask = np.zeros((len(mats), abi.GRAD_SLOTS), bool)
    for i, m in enumerate(mats):
        row = occupants.MATERIAL_BY_ID.get(m.model)
        # an emitter's record is a light's; a model with an IOR parameter is live only
        # where a region uses it (the IOR is a region row)
        if row is not None and not (m.flags & abi.MATF_EMISSIVE) and not (row.grad_ior and i not in used):
            if row.grad_color:
                mask[i, abi.GRAD_COLOR_R:abi.GRAD_COLOR_B + 1] = True
            if row.grad_alpha:
                mask[i, abi.GRAD_ALPHA] = True
            if row.grad_ior:
                mask[i, abi.GRAD_IOR] = True
        if m.flags & abi.MATF_MEDIUM:
            mask[i, abi.GRAD_SIGMA_T] = True
            mask[i, abi.GRAD_MEDIUM_ALBEDO] = True
            if m.flags & abi.MATF_SCATTERING:
                mask[i, abi.GRAD_HG_G] = True
    return mask


def param_table(packed):
    """(n_materials, GRAD_SLOTS) float64 parameter values (0 in unused slots)."""
    mats = _materials(packed)
    regs = _regions(packed)
    ior = {}
    for r in regs:
        ior.setdefault(r.material, r.ior)
    out = np.zeros((len(mats), abi.GRAD_SLOTS), np.float64)
    for i, m in enumerate(mats):
        out[i, 0:3] = list(_color(m))[:3]
        out[i, abi.GRAD_ALPHA] = m.alpha
        out[i, abi.GRAD_IOR] = ior.get(i, 1.0)
        st = m.sigma_a[0] + m.sigma_s[0]
        out[i, abi.GRAD_SIGMA_T] = st
        out[i, abi.GRAD_MEDIUM_ALBEDO] = m.sigma_s[0] / st if st > 0 else 0.0
        out[i, abi.GRAD_HG_G] = m.phase_g
    return out


def with_params(packed, table):
    """A copy of ``packed`` whose live parameters take the values of ``table``."""
    mask = live_mask(packed)
    out = copy.copy(packed)
    out.materials = packed.materials.copy()
    out.regions = packed.regions.copy()
    mats = _materials(out)
    regs = _regions(out)
    for i, m in enumerate(mats):
        row = table[i]
        if mask[i, 0]:
            setattr(m, _color_field(m), abi.F4(*(list(row[0:3]) + [0.0])))
        if mask[i, abi.GRAD_ALPHA]:
            m.alpha = float(row[abi.GRAD_ALPHA])
        if mask[i, abi.GRAD_SIGMA_T]:
            st, a = float(row[abi.GRAD_SIGMA_T]), float(row[abi.GRAD_MEDIUM_ALBEDO])
            m.sigma_a = abi.F4(*([(1.0 - a) * st] * 3 + [0.0]))
            m.sigma_s = abi.F4(*([a * st] * 3 + [0.0]))
        if mask[i, abi.GRAD_HG_G]:
            m.phase_g = float(row[abi.GRAD_HG_G])
    for r in regs:
        if r.material >= 0 and mask[r.material, abi.GRAD_IOR]:
            r.ior = float(table[r.material, abi.GRAD_IOR])
    return out


def l2_loss(image, target):
    """Mean over pixels and channels of (image - target)^2, and its derivative."""
    d = image.astype(np.float64) - target.astype(np.float64)
    n = d.size
    return float((d * d).sum() / n), (2.0 / n) * d
