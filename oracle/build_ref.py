"""Build ``oracle/_ref/``: the reference's own generated programs compiled for the host.

TEST INFRASTRUCTURE ONLY (the oracle's checker build; the product never links it).

Recipe: extract the assembled GLSL programs from the reference's snapshot file
(``extract_snapshots.py``), translate each to C++ (``glsl2cpp.py``) and compile it
with g++ against ``glsl_compat.hpp`` into ``oracle/_ref/<case>.so``.  Outputs go
only into ``oracle/_ref/`` (git-ignored; it travels with the working tree to the
GPU host, where the reference sources are absent).

Programs that read filtered textures (``texture()``) or write several render
targets are not translatable by the compat layer and are recorded as not built.

Usage: python oracle/build_ref.py [REFERENCE_ROOT] [--all]
"""
import concurrent.futures as cf
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import extract_snapshots  # noqa: E402
import glsl2cpp  # noqa: E402

OUT = os.path.join(HERE, "_ref")

# The analytic-scene cases the tests use (no data textures, no filtered lookups).
DEFAULT_CASES = [
    "cornell_area_glass_pt_mis", "cornell_area_glass_pt_nee", "cornell_area_glass_pt",
    "cornell_area_pt_mis", "furnace_sky_pt_mis", "furnace_sky_pt_nee", "furnace_no_direct",
    "eta_witness", "slab_witness", "fogcube_witness", "fog_area_pt_mis", "fog_area_pt_nee",
    "haze_pt_nee", "haze_pt", "furnace_scatter_witness", "orb_pt_nee", "orb_pt",
    "veach_mis", "two_light_power", "two_light_uniform", "cornell_glass", "submerged_witness",
]


def _compile(case, src_path):
    cpp = os.path.join(OUT, case + ".cpp")
    so = os.path.join(OUT, case + ".so")
    with open(src_path, encoding="utf-8") as f:
        text = f.read()
    with open(cpp, "w", encoding="utf-8") as f:
        f.write(glsl2cpp.translate(text, "p_" + case))
    cmd = ["g++", "-std=c++20", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-I" + HERE, cpp, "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return case, r.returncode == 0, r.stderr[-2000:]


# Where the reference checkout is read from (this build recipe's one default; the
# PTR_REFERENCE_DIR environment variable or the first argument overrides it).
REFERENCE_DIR = os.environ.get("PTR_REFERENCE_DIR", "/root/reference")


def build(ref_root=None, all_cases=False, jobs=None):
    ref_root = ref_root or REFERENCE_DIR
    snap = os.path.join(ref_root, extract_snapshots.SNAP_REL)
    if not os.path.exists(snap):
        return None
    os.makedirs(os.path.join(OUT, "glsl"), exist_ok=True)
    index = {}
    todo = []
    for name, rid, frag, meta in extract_snapshots.extract(snap):
        case = extract_snapshots.slug(name)
        path = os.path.join(OUT, "glsl", case + ".glsl")
        with open(path, "w", encoding="utf-8") as f:
            f.write(frag)
        index[case] = {"case": name, "renderer": rid, "built": False, **meta}
        if all_cases or case in DEFAULT_CASES:
            so = os.path.join(OUT, case + ".so")
            if os.path.exists(so) and os.path.getmtime(so) > max(os.path.getmtime(path) - 1e9, 0) \
                    and os.path.getmtime(so) >= os.path.getmtime(os.path.join(HERE, "glsl_compat.hpp")) \
                    and os.path.getmtime(so) >= os.path.getmtime(os.path.join(HERE, "glsl2cpp.py")):
                index[case]["built"] = True
                continue
            todo.append((case, path))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for case, ok, err in ex.map(lambda a: _compile(*a), todo):
            index[case]["built"] = ok
            if not ok:
                index[case]["error"] = err
    with open(os.path.join(OUT, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)
    return index


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    idx = build(args[0] if args else None, all_cases="--all" in sys.argv)
    if idx is None:
        print("reference snapshot not found; oracle/_ref not built")
    else:
        ok = sum(1 for v in idx.values() if v["built"])
        print(f"oracle/_ref: {ok} programs built of {len(idx)} extracted")
