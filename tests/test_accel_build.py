"""Host builders (binary SAH BVH, compressed wide BVH) — the reference's accel gates.

Restates the structure and traversal gates of the reference's tests/components/cwbvh.test.ts
(every item exactly once, leaf caps, conservative quantization, walk == brute force on
seeded sphere clouds, octant pruning, coincident centroids, 50k stack depth) and the
binary-tree invariants, against the builders compiled into libptx_rt.so (host code,
no GPU).  The walk below is a float64 transcription of the reference's cwbvhNearestRef
(src/components/accel/cwbvh/cwbvh.ts:429-502).
"""
import ctypes as C
import math
import struct

import numpy as np
import pytest

from pathtracerglsl_b200 import build

PAD = 1.00000024


@pytest.fixture(scope="module")
def lib():
    build.build()
    lb = C.CDLL(build.LIB)
    lb.ptr_build_bvh.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lb.ptr_build_cwbvh.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                                   C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return lb


def lcg(seed):
    s = seed & 0xFFFFFFFF

    def nxt():
        nonlocal s
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        return s / 4294967296.0
    return nxt


def sphere_cloud(n, seed, extent=10.0):
    rnd = lcg(seed)
    c = np.zeros((n, 3))
    r = np.zeros(n)
    for i in range(n):
        c[i] = [(rnd() * 2 - 1) * extent, (rnd() * 2 - 1) * extent, (rnd() * 2 - 1) * extent]
        r[i] = 0.05 + rnd() * 0.4
    boxes = np.concatenate([c - r[:, None], c + r[:, None]], axis=1)
    return np.ascontiguousarray(boxes), c, r


def build_bvh(lib, boxes, leaf=2, always=False):
    n = len(boxes)
    cnt, depth = C.c_int(), C.c_int()
    lib.ptr_build_bvh(boxes.ctypes.data, n, leaf, int(always), None, 0, None, C.byref(cnt), C.byref(depth))
    nodes = np.zeros((max(cnt.value, 1), 8), np.float32)
    order = np.zeros(max(n, 1), np.uint32)
    assert lib.ptr_build_bvh(boxes.ctypes.data, n, leaf, int(always), nodes.ctypes.data, cnt.value, order.ctypes.data,
                             C.byref(cnt), C.byref(depth)) == 0
    return nodes[:cnt.value], order[:n], depth.value


def build_cw(lib, boxes, c_prim=0.3):
    n = len(boxes)
    cnt, depth = C.c_int(), C.c_int()
    assert lib.ptr_build_cwbvh(boxes.ctypes.data, n, c_prim, None, 0, None, C.byref(cnt), C.byref(depth)) == 0
    nodes = np.zeros((max(cnt.value, 1), 20), np.uint32)
    order = np.zeros(max(n, 1), np.uint32)
    assert lib.ptr_build_cwbvh(boxes.ctypes.data, n, c_prim, nodes.ctypes.data, cnt.value, order.ctypes.data,
                               C.byref(cnt), C.byref(depth)) == 0
    return nodes[:cnt.value], order[:n], depth.value


def bits_float(u):
    return struct.unpack("<f", struct.pack("<I", int(u) & 0xFFFFFFFF))[0]


def decode(nodes, i):
    w = nodes[i]
    meta = [(int(w[6 + k // 4]) >> (8 * (k % 4))) & 0xFF for k in range(8)]
    qlo, qhi = [0] * 24, [0] * 24
    for ww in range(6):
        dst = qlo if ww < 3 else qhi
        off = (ww % 3) * 8
        for k in range(4):
            dst[off + k] = (int(w[8 + 2 * ww]) >> (8 * k)) & 0xFF
            dst[off + 4 + k] = (int(w[9 + 2 * ww]) >> (8 * k)) & 0xFF
    e = int(w[3])
    return {"p": [bits_float(w[0]), bits_float(w[1]), bits_float(w[2])],
            "scale": [bits_float((e & 0xFF) << 23), bits_float(((e >> 8) & 0xFF) << 23), bits_float(((e >> 16) & 0xFF) << 23)],
            "imask": (e >> 24) & 0xFF, "child": int(w[4]), "prim": int(w[5]), "meta": meta, "qlo": qlo, "qhi": qhi}


def popc8(v):
    return bin(v & 0xFF).count("1")


def msb(v):
    return v.bit_length() - 1


def cw_nearest(nodes, order, ro, rd, item_test):
    """float64 walk of cwbvhNearestRef (octant order, group stack, quantized slabs)."""
    tmax, best, visited = math.inf, -1, 0
    if len(nodes) == 0:
        return -1, math.inf, 0
    oct_ = (1 if rd[0] < 0 else 0) | (2 if rd[1] < 0 else 0) | (4 if rd[2] < 0 else 0)
    octinv = 7 - oct_
    safe = [(-1e-20 if d < 0 else 1e-20) if abs(d) < 1e-20 else d for d in rd]
    inv = [1.0 / d for d in safe]
    stack = []
    g_base, g_hits, g_imask = 0, 1 << (octinv & 7), 1
    while True:
        if g_hits == 0:
            if not stack:
                break
            g_base, g_hits, g_imask = stack.pop()
            continue
        bit = msb(g_hits)
        g_hits &= ~(1 << bit)
        slot = (bit ^ octinv) & 7
        child = g_base + popc8(g_imask & ((1 << slot) - 1))
        if g_hits:
            stack.append((g_base, g_hits, g_imask))
        visited += 1
        nd = decode(nodes, child)
        dq = [nd["scale"][a] * inv[a] for a in range(3)]
        oq = [(nd["p"][a] - ro[a]) * inv[a] for a in range(3)]
        hits = 0
        leaf_bits = 0
        for s in range(8):
            m = nd["meta"][s]
            if m == 0:
                continue
            tn, tf = 0.0, tmax
            for a in range(3):
                lo = nd["qlo"][8 * a + s] * dq[a] + oq[a]
                hi = nd["qhi"][8 * a + s] * dq[a] + oq[a]
                tn = max(tn, min(lo, hi))
                tf = min(tf, max(lo, hi))
            tf *= PAD
            if tf < tn:
                continue
            if (m & 0xE0) == 0x20 and (m & 0x1F) >= 24:
                hits |= 1 << ((((m & 0x1F) - 24) ^ octinv) & 7)
            else:
                leaf_bits |= (m >> 5) << (m & 0x1F)
        while leaf_bits:
            ib = msb(leaf_bits)
            leaf_bits &= ~(1 << ib)
            item = int(order[nd["prim"] + ib])
            t = item_test(item, tmax)
            if t < tmax:
                tmax, best = t, item
        if hits:
            g_base, g_hits, g_imask = nd["child"], hits, nd["imask"]
        else:
            g_hits = 0
    return best, tmax, visited


def ray_sphere(ro, rd, c, rad):
    o = [ro[k] - c[k] for k in range(3)]
    b = o[0] * rd[0] + o[1] * rd[1] + o[2] * rd[2]
    cc = o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - rad * rad
    disc = b * b - cc
    if disc < 0:
        return math.inf
    s = math.sqrt(disc)
    t0, t1 = -b - s, -b + s
    if t0 > 1e-4:
        return t0
    if t1 > 1e-4:
        return t1
    return math.inf


@pytest.mark.parametrize("n", [1, 2, 3, 7, 8, 25, 500])
def test_cwbvh_every_item_once_and_caps(lib, n):
    boxes, c, r = sphere_cloud(n, 1000 + n)
    nodes, order, depth = build_cw(lib, boxes)
    assert sorted(order.tolist()) == list(range(n))
    for i in range(len(nodes)):
        nd = decode(nodes, i)
        items = 0
        for s in range(8):
            m = nd["meta"][s]
            if m == 0 or ((m & 0xE0) == 0x20 and (m & 0x1F) >= 24):
                continue
            cnt = bin(m >> 5).count("1")
            assert 1 <= cnt <= 3
            items += cnt
        assert items <= 24


@pytest.mark.parametrize("n", [25, 500])
def test_cwbvh_quantized_boxes_contain_their_items(lib, n):
    """Conservative quantization: every decoded child box (float32 decode p + q*2^e)
    contains every item box below it."""
    boxes, c, r = sphere_cloud(n, 2000 + n)
    nodes, order, depth = build_cw(lib, boxes)

    def items_below(i):
        nd = decode(nodes, i)
        out = []
        ci = 0
        for s in range(8):
            m = nd["meta"][s]
            if m == 0:
                continue
            if (m & 0xE0) == 0x20 and (m & 0x1F) >= 24:
                sub = items_below(nd["child"] + popc8(nd["imask"] & ((1 << s) - 1)))
            else:
                off = m & 0x1F
                sub = [int(order[nd["prim"] + off + k]) for k in range(bin(m >> 5).count("1"))]
            for a in range(3):
                lo = np.float32(np.float32(nd["p"][a]) + np.float32(nd["qlo"][8 * a + s]) * np.float32(nd["scale"][a]))
                hi = np.float32(np.float32(nd["p"][a]) + np.float32(nd["qhi"][8 * a + s]) * np.float32(nd["scale"][a]))
                for it in sub:
                    assert lo <= boxes[it, a] and hi >= boxes[it, 3 + a]
            out += sub
            ci += 1
        return out

    assert sorted(items_below(0)) == list(range(n))


@pytest.mark.parametrize("n,seed", [(50, 11), (300, 12), (1000, 13)])
def test_cwbvh_walk_equals_brute_force(lib, n, seed):
    boxes, c, r = sphere_cloud(n, seed)
    nodes, order, depth = build_cw(lib, boxes)
    rnd = lcg(seed * 7 + 1)
    hits = 0
    for _ in range(200):
        ro = [(rnd() * 2 - 1) * 25, (rnd() * 2 - 1) * 25, (rnd() * 2 - 1) * 25]
        j = int(math.floor(rnd() * n))
        d = [c[j, k] + (rnd() * 2 - 1) * r[j] * 2 - ro[k] for k in range(3)]
        ln = math.hypot(*d) or 1.0
        d = [x / ln for x in d]
        bt, bi = math.inf, -1
        for i in range(n):
            t = ray_sphere(ro, d, c[i], r[i])
            if t < bt:
                bt, bi = t, i
        item, t, _ = cw_nearest(nodes, order, ro, d, lambda it, tm: (lambda tt: tt if tt < tm else math.inf)(ray_sphere(ro, d, c[it], r[it])))
        assert item == bi
        if bi >= 0:
            assert abs(t - bt) < 1e-9
            hits += 1
    assert hits > 20


def test_cwbvh_octant_order_prunes(lib):
    n = 512
    c = np.zeros((n, 3))
    c[:, 0] = np.arange(n) * 2.0
    r = np.full(n, 0.5)
    boxes = np.ascontiguousarray(np.concatenate([c - 0.5, c + 0.5], axis=1))
    nodes, order, depth = build_cw(lib, boxes)
    item, t, visited = cw_nearest(nodes, order, [-5, 0, 0], [1, 0, 0],
                                  lambda it, tm: (lambda tt: tt if tt < tm else math.inf)(ray_sphere([-5, 0, 0], [1, 0, 0], c[it], r[it])))
    assert item == 0
    assert visited < len(nodes) / 4


def test_cwbvh_coincident_centroids(lib):
    same = np.ascontiguousarray(np.tile([-1.0, -1, -1, 1, 1, 1], (4, 1)))
    nodes, order, _ = build_cw(lib, same)
    assert sorted(order.tolist()) == [0, 1, 2, 3]
    boxes, _, _ = sphere_cloud(1000, 77)
    boxes[1:6] = boxes[0]
    nodes, order, _ = build_cw(lib, np.ascontiguousarray(boxes))
    assert sorted(order.tolist()) == list(range(1000))


def test_cwbvh_depth_50k(lib):
    boxes, _, _ = sphere_cloud(50_000, 7)
    nodes, order, depth = build_cw(lib, boxes)
    assert depth < 24 // 2


def test_binary_bvh_invariants(lib):
    boxes, c, r = sphere_cloud(2000, 5)
    nodes, order, depth = build_bvh(lib, boxes, leaf=2)
    assert sorted(order.tolist()) == list(range(2000))
    seen = np.zeros(2000, int)

    def visit(i, lo, hi):
        n0 = nodes[i]
        mn, mx = n0[0:3], n0[4:7]
        assert (mn >= lo - 1e-6).all() and (mx <= hi + 1e-6).all()
        if n0[3] >= 0:
            cnt, off = int(n0[3]), int(n0[7])
            for k in range(off, off + cnt):
                it = order[k]
                seen[it] += 1
                assert (np.float32(boxes[it, 0:3]) >= mn).all() and (np.float32(boxes[it, 3:6]) <= mx).all()
        else:
            visit(i + 1, mn, mx)
            visit(int(n0[7]), mn, mx)

    visit(0, nodes[0][0:3], nodes[0][4:7])
    assert (seen == 1).all()
    assert depth < 64
