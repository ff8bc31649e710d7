"""Generate the golden fixtures of the reference's own programs (tests/golden/ref_images.npz).

Run here, where the reference is mounted: it builds oracle/_ref (the reference's snapshot
programs compiled on the host) and records, for every witness case of tests/ref_scenes.py,
the per-pixel mean of a small seeded render (24x24, 8 spp, salt 7) together with the
camera parameters it was bound with.  The CPU tests compare the oracle against these
fixtures, so the pin holds on machines without the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import build_ref  # noqa: E402
import ref_harness  # noqa: E402
import ref_scenes  # noqa: E402

W = H = 24
SPP = 8
SALT = 7


def camera_params(case):
    """Camera of each case: the snapshot program's parameter defaults, posed the way the
    reference's witness registry poses the scene (tests/witnesses/index.ts posed(...))."""
    p = ref_harness.RefProgram(case)
    cam = {k: v for k, v in p.defaults().items() if k.startswith("camera.")}
    scene, st = ref_scenes.CASES[case]
    c = st["measurement"].get("camera", {})
    if case.startswith("cornell") or case.startswith("fog_area"):
        cam["camera.position"], cam["camera.target"] = [0, 1, 4], [0, 1, 0]
    if "position" in c:
        cam["camera.position"], cam["camera.target"] = c["position"], c["target"]
    return cam


def main():
    build_ref.build(sys.argv[1] if len(sys.argv) > 1 else None)   # default: build_ref.REFERENCE_DIR
    out = {}
    for case in ref_scenes.CASES:
        cam = camera_params(case)
        prog = ref_harness.RefProgram(case)
        prog.bind(W, H, salt=SALT, params=cam)
        mean, _ = prog.stats(W, H, SPP)
        out[case] = mean.astype(np.float64)
        out[case + "__camera"] = np.array([*cam["camera.position"], *cam["camera.target"], cam["camera.fov"]])
    np.savez_compressed(os.path.join(HERE, "ref_images.npz"), W=W, H=H, SPP=SPP, SALT=SALT, **out)
    print("wrote", len(ref_scenes.CASES), "cases")


if __name__ == "__main__":
    main()
