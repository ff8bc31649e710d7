"""The reference's packed scene-data channels (rail v2) as this library's packer writes
them (pathtracerglsl_b200/rails.py), checked on the CPU against the ledger's rules
(src/components/data/ledger.ts:121-183, src/components/data/pack.ts): regions in ledger
order, disjoint, padded to their declared bounds, whole 4096-texel rows; payloads at
their bases; the BVH and TLAS node regions walk to every item exactly once."""
import numpy as np

from pathtracerglsl_b200 import _native, abi, rails, scenes
from pathtracerglsl_b200.compiler import Compiler


def test_layout_follows_the_ledger_order():
    totals, ms, bs, ls = rails.plan_layout([(10, 16), (4, 2)], [(5, 2), (3, 1)], [(1, 4, 2)])
    assert ms == [{"vbase": 0, "tbase": 0, "nbase": 0}, {"vbase": 10, "tbase": 16, "nbase": 2 * 31}]
    assert bs == [{"placements_base": 0, "tlas_base": 62 + 6}, {"placements_base": 10, "tlas_base": 68 + 18}]
    assert ls == [{"mesh": 1, "wpos_base": 14, "cdf_base": 13}]
    assert totals == {"vertices": 18, "indices": 18, "nodes": 86 + 10, "records": 15}
    assert rails.node_texel_bound(0) == 0 and rails.node_texel_bound(1) == 2
    assert len(rails.alloc_channel(0)) == 4096 * 4 and len(rails.alloc_channel(4097)) == 2 * 4096 * 4


def _walk(nodes, base, n_items):
    """Leaf items reached from the root of a bvh.ts node region."""
    q = nodes.reshape(-1, 4)
    seen, stack = [], [0]
    while stack:
        i = stack.pop()
        a, b = q[base + 2 * i][3], q[base + 2 * i + 1][3]
        if a >= 1:
            seen.extend(range(int(b), int(b) + int(a)))
        else:
            stack += [int(b), i + 1]
    return sorted(seen) == list(range(n_items))


def test_packer_writes_every_tenant_at_its_base():
    sc, st, _ = scenes.mesh_scene(level=2, instances=5, env_size=(16, 8))
    _, pk = Compiler().compile(sc, st)
    pr = rails.pack(pk, _native.load())
    for ch in (pr.vertices, pr.indices, pr.nodes, pr.records):
        assert len(ch) % (4096 * 4) == 0
    for m, mesh in zip(pr.meshes, pk.meshes):
        pos = np.asarray(mesh["positions"], np.float32).reshape(-1, 3)
        idx = np.asarray(mesh["indices"], np.uint32).reshape(-1, 3)
        v = pr.vertices.reshape(-1, 4)[m["vbase"]:m["vbase"] + len(pos)]
        np.testing.assert_array_equal(v[:, :3], pos)
        assert (v[:, 3] == 0).all()
        t = pr.indices.reshape(-1, 4)[m["tbase"]:m["tbase"] + len(idx)]
        np.testing.assert_array_equal(t[:, :3].astype(np.uint32), idx[m["tri_order"]])
        assert sorted(m["tri_order"]) == list(range(len(idx)))
        assert m["node_count"] * 2 <= rails.node_texel_bound(len(idx))
        assert _walk(pr.nodes, m["nbase"], len(idx))
    for b, batch in zip(pr.batches, pk.batches):
        n = len(batch["placements"]) // 8
        assert b["placement_texels"] == (2 if batch["prototype_shape"] == abi.SHAPE_MESH else 1)
        rec = pr.records.reshape(-1, 4)[b["placements_base"]:b["placements_base"] + 2 * n].reshape(n, 8)
        np.testing.assert_array_equal(rec, np.asarray(batch["placements"], np.float32).reshape(n, 8)[b["inst_order"]])
        assert _walk(pr.nodes, b["tlas_base"], n)


def test_mesh_light_tables_follow_leaf_order():
    sc, st = scenes.cornell_mesh_light(direct="mis", emitter="sphere")
    _, pk = Compiler().compile(sc, st)
    pr = rails.pack(pk, _native.load())
    assert len(pr.mesh_lights) == 1
    l = pr.mesh_lights[0]
    m = pr.meshes[l["mesh"]]
    cdf = pr.records.reshape(-1, 4)[l["cdf_base"]:l["cdf_base"] + m["tri_count"], 0]
    assert cdf[-1] == 1.0 and (np.diff(cdf) >= 0).all() and cdf[0] > 0
    wpos = pr.vertices.reshape(-1, 4)[l["wpos_base"]:l["wpos_base"] + m["vertex_count"], :3]
    np.testing.assert_array_equal(wpos, np.asarray(pk.meshes[l["mesh"]]["positions"], np.float32).reshape(-1, 3))
