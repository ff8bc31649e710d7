"""The multi-GPU replica plumbing, as two gloo ranks on CPU (no GPU): distinct sample
streams per rank, max-over-ranks timing and the float64 film combination."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from pathtracerglsl_b200.replicas import Replicas
    r = Replicas.from_env(backend="gloo", timeout_s=60)
    try:
        salt = r.salt(1)
        t = r.max(10.0 + rank)            # each rank's "device time"
        r.barrier()
        # rank k's film: 2 samples of value k+1 per pixel
        s = np.full((2, 3, 3), 2.0 * (rank + 1))
        q = np.full((2, 3, 3), 2.0 * (rank + 1) ** 2)
        mean, sumsq, n = r.combine_film(s, q, 2.0)
        out.put((rank, salt, t, float(mean.mean()), float(n)))
    finally:
        r.close()


def test_two_gloo_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] != res[1][1]                       # decorrelated streams
    assert res[0][2] == res[1][2] == 11.0               # max over ranks
    assert res[0][3] == res[1][3] == pytest.approx(1.5)  # (2*1 + 2*2) / 4 samples
    assert res[0][4] == res[1][4] == 4.0


def test_single_process_is_a_noop():
    from pathtracerglsl_b200.replicas import Replicas
    r = Replicas.from_env()
    assert r.world == 1 and r.salt(5) == 5 and r.max(3.0) == 3.0
    m, _, n = r.combine_film(np.ones((2, 2, 3)) * 4.0, np.ones((2, 2, 3)), 2.0)
    assert n == 2.0 and np.allclose(m, 2.0)
