"""Make ``jh_cie1931_d65_subset.npz``: the part of the reference's spectral model this
package's workloads and tests read.

The reference ships its spectral model (version jh-cie1931-d65-v1) as two float32 assets in
src/components/color/spectral/data/: curves.bin (CIE 1931 x, y, z and D65 at 5 nm from
360 nm in row 0, the 64 intensity nodes in row 1) and coefficients.bin (the 3 x 64^3
Jakob-Hanika atlas, 12.6 MB), plus its XYZ -> linear-sRGB matrix in data.ts.  This script
copies the curves, the nodes and the matrix, and only those atlas nodes the lookups of
COLOURS read (8 per non-grey colour), so the package carries a few KB instead of 12 MB.
Colours outside the subset need the full assets (SpectralModel.from_assets).

Usage: python pathtracerglsl_b200/data/make_spectral_subset.py [REFERENCE_ROOT]
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from pathtracerglsl_b200.spectral import SpectralModel  # noqa: E402

# (rgb, kind): kind 'r' reflectance, 'c' coefficient (sigma / emission: rgb / (2 max rgb))
COLOURS = [
    ((0.5, 1.0, 2.0), "c"), ((0.05, 0.1, 0.2), "c"), ((0.45, 0.9, 1.8), "c"),   # media workload sigma_t, a, s
    ((0.7, 0.5, 0.3), "r"), ((0.75, 0.25, 0.25), "r"), ((0.25, 0.75, 0.25), "r"),
    ((0.9, 0.6, 0.3), "r"), ((0.3, 0.6, 0.9), "r"), ((0.2, 0.4, 0.8), "c"), ((1.0, 0.8, 0.6), "c"),
    ((0.8, 0.3, 0.1), "c"),
]


def main(ref_root=None):
    """ref_root: the reference checkout (default: the PTR_REFERENCE_DIR environment variable)."""
    ref_root = ref_root or os.environ.get("PTR_REFERENCE_DIR")
    if not ref_root:
        raise SystemExit("usage: make_spectral_subset.py <reference checkout> (or set PTR_REFERENCE_DIR)")
    data_dir = os.path.join(ref_root, "src/components/color/spectral/data")
    model = SpectralModel.from_assets(data_dir)
    idx = set()
    for rgb, kind in COLOURS:
        if kind == "c":
            s = 2.0 * max(rgb)
            rgb = tuple(np.float32(v) / np.float32(s) for v in rgb)
        idx.update(model.nodes_of(rgb))
    idx = sorted(idx)
    atlas = np.fromfile(os.path.join(data_dir, "coefficients.bin"), dtype="<f4").reshape(-1, 4)
    coef = atlas[idx, :3]
    text = open(os.path.join(ref_root, "src/components/color/spectral/data.ts")).read()
    block = re.search(r'"xyzToRGB":\s*\[(.*?)\]\s*\]', text, re.S).group(1)
    m = np.array([float(v) for v in re.findall(r"-?\d+\.\d+(?:e-?\d+)?", block)]).reshape(3, 3)
    np.savez(os.path.join(HERE, "jh_cie1931_d65_subset.npz"), curves=model.curves, z_nodes=model.z_nodes,
             xyz_to_rgb=m, node_index=np.array(idx, np.int64), node_coef=coef.astype(np.float32))
    print(f"{len(idx)} atlas nodes for {len(COLOURS)} colours")


if __name__ == "__main__":
    main(*sys.argv[1:])
