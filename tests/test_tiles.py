"""Tiled renders on the CPU: the tile plan (the cases of the reference's
tests/app/tiling.test.ts) and a tile of the oracle against the same pixels of its
full-frame render, bit for bit.  The RNG seeds with the global pixel and the camera maps
film points through the full image size (pinhole.glsl:6), so a tile computes exactly
what the full render computes there."""
import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler
from pathtracerglsl_b200.engine import TILE_ALIGN, plan_tiles


@pytest.mark.parametrize("w,h,size", [(1030, 700, 512), (64, 64, 64), (1, 1, 1024), (4000, 2250, 1000)])
def test_plan_covers_the_image_exactly_once(w, h, size):
    plan = plan_tiles(w, h, size)
    hits = np.zeros((h, w), np.uint8)
    for t in plan["tiles"]:
        hits[t["y"]:t["y"] + t["height"], t["x"]:t["x"] + t["width"]] += 1
    assert (hits == 1).all()
    assert len(plan["tiles"]) == plan["cols"] * plan["rows"]


def test_plan_offsets_sit_on_the_alignment_grid():
    plan = plan_tiles(1030, 700, 500)
    assert plan["size"] == 512
    assert all(t["x"] % TILE_ALIGN == 0 and t["y"] % TILE_ALIGN == 0 for t in plan["tiles"])


def test_plan_cuts_the_last_column_and_the_top_row():
    plan = plan_tiles(1030, 700, 512)
    assert (plan["cols"], plan["rows"]) == (3, 2)
    at = {(t["col"], t["row"]): t for t in plan["tiles"]}
    assert at[0, 1] == dict(col=0, row=1, x=0, y=0, width=512, height=512)
    assert at[2, 1] == dict(col=2, row=1, x=1024, y=0, width=6, height=512)
    assert at[0, 0] == dict(col=0, row=0, x=0, y=512, width=512, height=188)
    assert (plan["tiles"][0]["col"], plan["tiles"][0]["row"]) == (0, 0)


def test_plan_rejects_bad_sizes():
    for args, name in (((0, 10, 64), "width"), ((10, 10.5, 64), "height"), ((10, 10, 0), "tileSize")):
        with pytest.raises(ValueError, match=name):
            plan_tiles(*args)


def test_oracle_tiles_reassemble_the_full_frame(oracle_lib):
    sc, st = scenes.cornell(direct="mis")
    r, pk = Compiler().compile(sc, st)
    W, H, spp = 150, 100, 2
    full = oracle_lib.render(pk, r, W, H, spp, salt=9, keep_samples=True)
    stitched = np.zeros((spp, H, W, 3), np.float32)
    for t in plan_tiles(W, H, 64)["tiles"]:
        o = oracle_lib.render(pk, r, t["width"], t["height"], spp, salt=9, keep_samples=True,
                              pixel_offset=(t["x"], t["y"]), image_size=(W, H))
        stitched[:, t["y"]:t["y"] + t["height"], t["x"]:t["x"] + t["width"]] = o["samples"]
    np.testing.assert_array_equal(stitched, full["samples"])
