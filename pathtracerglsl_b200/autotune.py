"""Autotuner of the wavefront's launch knobs: path-pool capacity, block size, the
occupant-sort bucket count and the ray-coherence queue order (ptr_tuning).  No counterpart
in the reference (its WebGL engine has no such knobs).

``tune(engine, render, candidates)`` times ``render()`` under every candidate on the
engine's context (device time through ptr_sync, best of ``repeats`` after one untimed
warm-up), keeps the fastest, applies it to the context and returns a record that
``save``/``load`` write to and read from a JSON file keyed by workload and GPU name.
"""
import itertools
import json
import os
import time

DEFAULT_CANDIDATES = [{"capacity": c, "block": b, "sort_buckets": k, "ray_sort": r}
                      for c, b, k, r in itertools.product((1 << 23, 1 << 24), (128, 256), (1, 8, 16), (0, 1))]
KNOBS = ("capacity", "block", "sort_buckets", "ray_sort")
DEFAULTS = {"capacity": 0, "block": 256, "sort_buckets": 1, "ray_sort": 0}


def tune(engine, render, candidates=None, repeats=1, budget_s=60.0, min_time_s=0.0):
    """Time render() under each candidate tuning; apply and return the best record.

    Each candidate runs `repeats` timed renders, and more while their total stays under
    `min_time_s` (short renders need many repetitions to separate candidates a few per
    cent apart); its time is the best single render."""
    candidates = list(candidates or DEFAULT_CANDIDATES)
    results = []
    t_start = time.perf_counter()
    for cand in candidates:
        cand = dict(DEFAULTS, **cand)
        engine.set_tuning(**cand)
        render()                       # warm-up: pool allocation, graph capture
        engine.sync()
        best = float("inf")
        spent = 0.0
        k = 0
        while k < max(1, repeats) or spent < min_time_s:
            t0 = time.perf_counter()
            render()
            engine.sync()
            dt = time.perf_counter() - t0
            best = min(best, dt)
            spent += dt
            k += 1
        results.append(dict(cand, ms=1000.0 * best))
        if time.perf_counter() - t_start > budget_s:
            break
    best = min(results, key=lambda r: r["ms"])
    engine.set_tuning(**{k: best[k] for k in KNOBS})
    return {"best": best, "results": results}


def gpu_name():
    try:
        import torch
        return torch.cuda.get_device_name(0)
    except Exception:   # no torch / no device: the record still keys by workload
        return "unknown"


def save(path, workload, record):
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data.setdefault(gpu_name(), {})[workload] = record
    with open(path, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)


def load(path, workload):
    """The recorded best tuning of a workload on this GPU, or None."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        data = json.load(f)
    rec = data.get(gpu_name(), {}).get(workload)
    return {k: rec["best"][k] for k in KNOBS if k in rec["best"]} if rec else None
