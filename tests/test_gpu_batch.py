"""Batched wavefront (ptr_render_batch) on the GPU.

The batched path draws the same counter-based random numbers per (job, pixel, sample)
as a plain one-job render, and both films add every pixel's samples in sample order, so
every job's film equals its plain film bit for bit.
Plain renders are checked against the oracle elsewhere; here one many-sphere job (the
region BVH dispatch) is also compared with the oracle directly.
"""
import os

import numpy as np
import pytest

from pathtracerglsl_b200 import scenes
from pathtracerglsl_b200.compiler import Compiler

pytestmark = pytest.mark.gpu


def _jobs(n, seed, max_spheres, res_cap, spp_cap):
    items, frames = [], []
    for k, (sc, st, (w, h, spp)) in enumerate(scenes.batch_scenes(n, seed, max_spheres)):
        r, pk = Compiler().compile(sc, st)
        items.append((r, pk))
        w = min(w, res_cap) - 8 * (k % 3)            # ragged sizes
        frames.append((w, w, min(spp, spp_cap), 0, 5 + k))
    return items, frames


def _check_batched_equals_plain(engine, items, frames):
    b = engine.batch(items)
    try:
        b.render(frames)
        batched = [b.read_export(j).copy() for j in range(len(b))]
        bvar = [b.read_export(j, "variance").copy() for j in range(len(b))]
        c = b.counters()
        assert c["paths"] == sum(f[0] * f[1] * f[2] for f in frames)
        b.render_plain(frames)
        for j in range(len(b)):
            plain = b.read_export(j)
            assert np.isfinite(batched[j]).all()
            np.testing.assert_array_equal(batched[j], plain)
            np.testing.assert_array_equal(bvar[j], b.read_export(j, "variance"))
        return b, batched
    except Exception:
        b.close()
        raise


def test_batch_equals_plain_per_job(engine):
    items, frames = _jobs(8, 3, 40, 48, 8)
    b, _ = _check_batched_equals_plain(engine, items, frames)
    b.close()


def test_batch_waves_split_jobs(engine, monkeypatch):
    """A small path pool: waves end inside jobs and jobs start inside waves."""
    monkeypatch.setenv("PTR_CAPACITY", "3000")
    items, frames = _jobs(5, 4, 12, 40, 4)
    b, _ = _check_batched_equals_plain(engine, items, frames)
    b.close()


def test_batch_accumulates_like_plain(engine):
    """Two batched calls (first_sample advancing, accumulate) equal one plain call of
    the summed spp."""
    items, frames = _jobs(3, 5, 10, 32, 4)
    b = engine.batch(items)
    try:
        b.render(frames)
        b.render([(w, h, spp, spp, salt) for (w, h, spp, _, salt) in frames])
        two = [b.read_export(j).copy() for j in range(len(b))]
        b.render_plain([(w, h, 2 * spp, 0, salt) for (w, h, spp, _, salt) in frames])
        for j in range(len(b)):
            np.testing.assert_array_equal(two[j], b.read_export(j))
    finally:
        b.close()


def test_batch_job_matches_oracle(engine, oracle_lib):
    """A 60-sphere job (region BVH) batched together with two small jobs, against the
    oracle's mean at the 3-sigma gate."""
    sc, st, _ = scenes.batch_scene(7, max_spheres=60)
    n_sph = len(sc["objects"]) - 5
    assert n_sph >= 8
    items = [Compiler().compile(sc, st)]
    frames = [(40, 40, 16, 0, 9)]
    for k in (11, 12):
        s2, t2, _ = scenes.batch_scene(k, max_spheres=6)
        items.append(Compiler().compile(s2, t2))
        frames.append((24, 24, 4, 0, 3))
    b = engine.batch(items)
    try:
        b.render(frames)
        m = b.read_export(0).astype(np.float64)
        r, pk = items[0]
        o = oracle_lib.render(pk, r, 40, 40, 16, salt=9)
        se = np.sqrt(2.0 * o["var"] / 16)
        ok = np.abs(m - o["mean"]) <= 3.0 * se + 1e-5
        assert ok.all(axis=-1).mean() >= 0.997
        # per-sample streams agree, so the means agree far below the noise
        assert np.abs(m - o["mean"]).mean() < 1e-3 * max(1e-3, o["mean"].mean())
    finally:
        b.close()


def test_batch_rejects_mixed_direct_lighting(engine):
    sc, st, _ = scenes.batch_scene(1, max_spheres=3)
    st2 = dict(st, id="x-nee", estimator=dict(st["estimator"], directLighting="nee"))
    items = [Compiler().compile(sc, st), Compiler().compile(sc, st2)]
    b = engine.batch(items)
    try:
        with pytest.raises(Exception, match="directLighting"):
            b.render([(16, 16, 1), (16, 16, 1)])
    finally:
        b.close()


def test_region_bvh_equals_the_linear_scan(engine, monkeypatch):
    """The region BVH (forced for 8+ bounded regions) returns the linear scan's hits: same
    nearest region, and on an exact tie the lower region index, so samples are identical."""
    sc, st, _ = scenes.batch_scene(7, max_spheres=60)
    assert len(sc["objects"]) - 5 >= 8
    r, pk = Compiler().compile(sc, st)
    out = []
    for minimum in ("1000000", "8"):
        monkeypatch.setenv("PTR_REGION_BVH_MIN", minimum)
        engine.register_scene(pk)
        engine.load_renderer(r)
        engine.select_renderer(r.id)
        engine.pin_reset_salt(6)
        engine.reset()
        out.append(engine.render_samples(40, 40, 4))
    np.testing.assert_array_equal(out[1], out[0])


def test_specialised_batch_equals_generic_and_plain(engine):
    """ptr_specialize_batch: the mix's union-census kernels render every job's film equal
    to the generic batched kernels and to the plain path; the progressive plain (one
    sample per launch, the reference's frame loop) folds the same samples."""
    items, frames = _jobs(6, 8, 30, 40, 6)
    b = engine.batch(items)
    try:
        b.render(frames)
        generic = [b.read_export(j).copy() for j in range(len(b))]
        secs = b.specialize()
        assert secs >= 0.0
        b.render(frames)
        for j in range(len(b)):
            np.testing.assert_allclose(b.read_export(j), generic[j], rtol=1e-9, atol=1e-12)
        b.render_plain(frames)
        for j in range(len(b)):
            np.testing.assert_allclose(b.read_export(j), generic[j], rtol=1e-9, atol=1e-12)
        b.render_progressive(frames)
        for j in range(len(b)):
            np.testing.assert_allclose(b.read_export(j), generic[j], rtol=1e-6, atol=1e-9)
    finally:
        b.close()
