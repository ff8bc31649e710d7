"""The reference's packed scene-data channels (rail v2) for a packed scene.

The reference's App packs a scene's array data into RGBA32F channels at the base texels
its ledger assigns (planDataLayout, src/components/data/ledger.ts:121-183; the writers of
src/components/data/pack.ts; executed by packSceneData, src/app/sceneData.ts:27).
``ptr_upload_scene_rails`` uploads such channels as they are.  This module produces them
from a ``PackedScene`` the way the App does, for the tenants the upload reads:

* geometry slots, one per mesh: the vertices (one vec3 texel each), the triangles in BVH
  leaf order (three vertex ids as exact floats per texel) and the binary BVH nodes (two
  texels each, region padded to 2 (2T - 1) texels); buildBVH (accel/bvh/bvh.ts:439-464)
  over the triangle boxes with leaf size 2, here by ``ptr_build_bvh``;
* instance batches: the placement records in TLAS leaf order (frame tier two texels, the
  params tier's folded (centre, radius) one texel) and the TLAS nodes (region padded to
  2 (2N - 1)); packInstanceBatch (intersection/instancing/instancing.ts:129-160);
* mesh lights: the world-position bake (vertices channel) and the area CDF in leaf order
  (records channel, .x); packMeshLight (lights/mesh/mesh.ts).

The optional tenants the ledger appends after these (the CWBVH twin, the object table,
the light tree, region materials) are not produced: this library builds or reads those
from the scene description.  Besides the channels it returns the leaf permutations
(``tri_order``, ``inst_order``) that make hit ids the caller's.
"""
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

DATA_TEX_WIDTH = 4096   # pack.ts DATA_TEX_WIDTH: texels per channel row
LEAF_SIZE = 2           # BVH_LEAF_SIZE / TLAS_LEAF_SIZE


def node_texel_bound(n):
    """ledger.ts nodeTexelBound: at most 2n - 1 nodes of two texels each."""
    return 2 * (2 * n - 1) if n > 0 else 0


def plan_layout(meshes, batches, mesh_lights):
    """planDataLayout for these tenants, in its order: geometry slots (vbase, tbase, nbase),
    then per batch its placements (records) and TLAS (nodes), then per mesh light its
    world positions (vertices) and CDF (records).

    meshes: [(vertex_count, tri_count)]; batches: [(instance_count, placement_texels)];
    mesh_lights: [(mesh, vertex_count, tri_count)].  Returns (totals, mesh slots, batch
    slots, light slots)."""
    v = t = n = r = 0
    mesh_slots = []
    for vc, tc in meshes:
        mesh_slots.append({"vbase": v, "tbase": t, "nbase": n})
        v += vc
        t += tc
        n += node_texel_bound(tc)
    batch_slots = []
    for count, texels in batches:
        slot = {"placements_base": r}
        r += texels * count
        slot["tlas_base"] = n
        n += node_texel_bound(count)
        batch_slots.append(slot)
    light_slots = []
    for mesh, vc, tc in mesh_lights:
        light_slots.append({"mesh": mesh, "wpos_base": v, "cdf_base": r})
        v += vc
        r += tc
    return {"vertices": v, "indices": t, "nodes": n, "records": r}, mesh_slots, batch_slots, light_slots


def alloc_channel(texels):
    """pack.ts allocChannel: a zero-filled channel of whole 4096-texel rows."""
    rows = max(1, math.ceil(max(1, texels) / DATA_TEX_WIDTH))
    return np.zeros(DATA_TEX_WIDTH * rows * 4, np.float32)


def _write_items(ch, base, items):
    """pack.ts writeItems: item k's components at texel base + k (the rest stay 0)."""
    items = np.asarray(items, np.float32)
    k = items.shape[1]
    view = ch.reshape(-1, 4)
    view[base:base + len(items), :k] = items


def _bvh(boxes, lib):
    """buildBVHNodesFlat over float64 boxes (6 per item), leaf size 2: (nodes, order)."""
    n = len(boxes)
    b = np.ascontiguousarray(boxes, np.float64)
    cnt, depth = C.c_int(), C.c_int()
    if lib.ptr_build_bvh(b.ctypes.data, n, LEAF_SIZE, 0, None, 0, None, C.byref(cnt), C.byref(depth)) != 0:
        raise RuntimeError("ptr_build_bvh failed")
    nodes = np.zeros(8 * cnt.value, np.float32)
    order = np.zeros(n, np.uint32)
    if lib.ptr_build_bvh(b.ctypes.data, n, LEAF_SIZE, 0, nodes.ctypes.data, cnt.value, order.ctypes.data,
                         C.byref(cnt), C.byref(depth)) != 0:
        raise RuntimeError("ptr_build_bvh failed")
    return nodes, order


def _to_world(pl, x, y, z):
    """World point of a prototype-local point under a placement (q, t_rigid, s): rotate by
    conj(q) the point s * local - t_rigid (the order of the library's own upload)."""
    qx, qy, qz, qw, tx, ty, tz, sc = (float(v) for v in pl)
    vx, vy, vz = sc * x - tx, sc * y - ty, sc * z - tz
    cx, cy, cz = -qx, -qy, -qz
    c1x, c1y, c1z = cy * vz - cz * vy + qw * vx, cz * vx - cx * vz + qw * vy, cx * vy - cy * vx + qw * vz
    c2x, c2y, c2z = cy * c1z - cz * c1y, cz * c1x - cx * c1z, cx * c1y - cy * c1x
    return vx + 2.0 * c2x, vy + 2.0 * c2y, vz + 2.0 * c2z


@dataclass
class PackedRails:
    """The channels (float32, four floats per texel) and the slot tables of a scene."""
    vertices: np.ndarray
    indices: np.ndarray
    nodes: np.ndarray
    records: np.ndarray
    meshes: list = field(default_factory=list)       # dicts: bases, counts, tri_order, tri_alpha
    batches: list = field(default_factory=list)      # dicts: bases, counts, placement_texels, inst_order
    mesh_lights: list = field(default_factory=list)  # dicts: mesh, wpos_base, cdf_base

    def struct(self, with_orders=True):
        """A ``ptr_rails`` pointing into this object's arrays (keep self alive).  Without
        orders, hit ids are leaf indices (the reference's own)."""
        r = abi.Rails()
        f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        r.vertices, r.vertices_texels = f(self.vertices), len(self.vertices) // 4
        r.indices, r.indices_texels = f(self.indices), len(self.indices) // 4
        r.nodes, r.nodes_texels = f(self.nodes), len(self.nodes) // 4
        r.records, r.records_texels = f(self.records), len(self.records) // 4
        self._mesh_arr = (abi.RailMesh * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            d = self._mesh_arr[i]
            d.vbase, d.tbase, d.nbase = m["vbase"], m["tbase"], m["nbase"]
            d.vertex_count, d.tri_count, d.node_count = m["vertex_count"], m["tri_count"], m["node_count"]
            order = m["tri_order"] if with_orders else None
            d.tri_order = order.ctypes.data_as(C.POINTER(C.c_uint32)) if order is not None else None
            alpha = m["tri_alpha"]
            if alpha is not None and not with_orders:   # alpha by leaf index
                alpha = m["tri_alpha_leaf"]
            d.tri_alpha = alpha.ctypes.data_as(C.POINTER(C.c_float)) if alpha is not None else None
        self._batch_arr = (abi.RailBatch * max(1, len(self.batches)))()
        for i, b in enumerate(self.batches):
            d = self._batch_arr[i]
            d.placements_base, d.tlas_base = b["placements_base"], b["tlas_base"]
            d.instance_count, d.node_count, d.placement_texels = b["instance_count"], b["node_count"], b["placement_texels"]
            order = b["inst_order"] if with_orders else None
            d.inst_order = order.ctypes.data_as(C.POINTER(C.c_uint32)) if order is not None else None
        self._light_arr = (abi.RailMeshLight * max(1, len(self.mesh_lights)))()
        for i, l in enumerate(self.mesh_lights):
            d = self._light_arr[i]
            d.mesh, d.wpos_base, d.cdf_base = l["mesh"], l["wpos_base"], l["cdf_base"]
        r.n_meshes, r.n_batches, r.n_mesh_lights = len(self.meshes), len(self.batches), len(self.mesh_lights)
        r.meshes, r.batches, r.mesh_lights = self._mesh_arr, self._batch_arr, self._light_arr
        self._struct = r
        return r


def pack(packed, lib):
    """The rail channels of a ``PackedScene`` as the reference's App packs them; ``lib`` is
    the loaded library (its host BVH builder)."""
    mesh_bvh = []
    for m in packed.meshes:
        pos = np.asarray(m["positions"], np.float32).reshape(-1, 3)
        idx = np.asarray(m["indices"], np.uint32).reshape(-1, 3)
        v = pos[idx].astype(np.float64)                      # (T, 3 vertices, xyz)
        boxes = np.concatenate([v.min(axis=1), v.max(axis=1)], axis=1)
        nodes, order = _bvh(boxes, lib)
        mesh_bvh.append((pos, idx, nodes, order))
    light_meshes = [int(l.p[0]) for l in (abi.Light * len(packed.lights)).from_buffer(packed.lights)
                    if l.kind == abi.LIGHT_MESH] if len(packed.lights) else []
    batch_tiers = [2 if b["prototype_shape"] == abi.SHAPE_MESH else 1 for b in packed.batches]
    totals, mslots, bslots, lslots = plan_layout(
        [(len(p), len(i)) for p, i, _, _ in mesh_bvh],
        [(len(b["placements"]) // 8, t) for b, t in zip(packed.batches, batch_tiers)],
        [(mi, len(mesh_bvh[mi][0]), len(mesh_bvh[mi][1])) for mi in light_meshes])
    ch = {k: alloc_channel(v) for k, v in totals.items()}
    out = PackedRails(ch["vertices"], ch["indices"], ch["nodes"], ch["records"])
    roots = []
    for (pos, idx, nodes, order), slot, m in zip(mesh_bvh, mslots, packed.meshes):
        _write_items(ch["vertices"], slot["vbase"], pos)
        _write_items(ch["indices"], slot["tbase"], idx[order].astype(np.float32))
        ch["nodes"].reshape(-1, 4)[slot["nbase"]:slot["nbase"] + len(nodes) // 4] = nodes.reshape(-1, 4)
        alpha = m.get("tri_alpha")
        out.meshes.append(dict(slot, vertex_count=len(pos), tri_count=len(idx), node_count=len(nodes) // 8,
                               tri_order=np.ascontiguousarray(order, np.uint32),
                               tri_alpha=None if alpha is None else np.ascontiguousarray(alpha, np.float32),
                               tri_alpha_leaf=None if alpha is None else np.ascontiguousarray(np.asarray(alpha, np.float32)[order])))
        roots.append((nodes[0:3].astype(np.float64), nodes[4:7].astype(np.float64)))
    for b, slot, tier in zip(packed.batches, bslots, batch_tiers):
        pl = np.asarray(b["placements"], np.float32).reshape(-1, 8)
        n = len(pl)
        boxes = np.zeros((n, 6))
        rec = np.zeros((n, 4 * tier), np.float32)
        for i in range(n):
            if tier == 2:
                lo, hi = roots[b["prototype_ref"]]
                corners = [_to_world(pl[i], hi[0] if k & 1 else lo[0], hi[1] if k & 2 else lo[1], hi[2] if k & 4 else lo[2])
                           for k in range(8)]
                boxes[i, :3] = np.min(corners, axis=0)
                boxes[i, 3:] = np.max(corners, axis=0)
                rec[i] = pl[i]
            else:   # params tier: the folded world (centre, radius)
                p = b["proto"]
                c = _to_world(pl[i], float(np.float32(p[0])), float(np.float32(p[1])), float(np.float32(p[2])))
                r = float(pl[i][7]) * float(np.float32(p[3]))
                boxes[i, :3] = [c[0] - r, c[1] - r, c[2] - r]
                boxes[i, 3:] = [c[0] + r, c[1] + r, c[2] + r]
                rec[i] = [c[0], c[1], c[2], r]
        nodes, order = _bvh(boxes, lib)
        base = slot["placements_base"]
        ch["records"].reshape(-1, 4)[base:base + n * tier] = rec[order].reshape(-1, 4)
        nb = slot["tlas_base"]
        ch["nodes"].reshape(-1, 4)[nb:nb + len(nodes) // 4] = nodes.reshape(-1, 4)
        out.batches.append(dict(slot, instance_count=n, node_count=len(nodes) // 8, placement_texels=tier,
                                inst_order=np.ascontiguousarray(order, np.uint32)))
    for lslot in lslots:
        pos, idx, _, order = mesh_bvh[lslot["mesh"]]
        _write_items(ch["vertices"], lslot["wpos_base"], pos)   # the mesh's world positions
        tri = pos[idx[order]].astype(np.float64)              # leaf order
        u, w = tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
        area = np.linalg.norm(np.cross(u, w), axis=1) / 2.0
        run = np.cumsum(area)   # sequential, like the packer's running sum
        acc = float(run[-1])
        cdf = (run / acc if acc > 0 else np.arange(1, len(area) + 1) / len(area)).astype(np.float32)
        cdf[-1] = 1.0
        ch["records"].reshape(-1, 4)[lslot["cdf_base"]:lslot["cdf_base"] + len(cdf), 0] = cdf
        out.mesh_lights.append(lslot)
    return out
