"""The multi-rank path on the host: two gloo ranks on CPU shard events, reduce a gradient
and take the maximum of their timings; the result must equal the one-process result.
(The GPUs of a multi-GPU job run the same code with NCCL.)"""
import os
import socket

import numpy as np
import pytest

from ppc_b200 import replicas as R
from ppc_b200 import types as T

EVENTS, GSIZE, SIZE = 7, 11, 5


def _bunches():
    b = np.concatenate([T.bunch_led([0, 0, 0, 0], [0, 0, 1], e, 100 * (e + 1), 1, ka=-1, up=0, fldr=-1)
                        for e in range(EVENTS) for _ in range(2)])
    return b


def _fake_gradient(bunches, observed, events):
    """Stands in for PPC.gradient: per-(event, DOM) charges from the bunches of each event,
    a Poisson log-likelihood and a gradient that depends on every event."""
    counts = np.zeros((events, GSIZE))
    for x in bunches:
        counts[x["q"]] += (np.arange(GSIZE) + 1) * int(x["num"]) % 13 + 1
    obs = np.asarray(observed, np.float64).reshape(events, GSIZE)
    ll = float(np.sum(obs * np.log(counts) - counts))
    w = (obs / counts - 1).sum(axis=1)
    g_be = np.outer(w, np.arange(1, SIZE + 1)).sum(axis=0)
    g_ba = np.outer(w ** 2, np.ones(SIZE)).sum(axis=0)
    return {"ll": ll, "g_be": g_be, "g_ba": g_ba, "counts": counts}


def _observed():
    return np.random.default_rng(1).poisson(20, (EVENTS, GSIZE)).astype(np.float32)


def _worker(rank, world, port, out):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = R.gradient_over_ranks(_fake_gradient, _bunches(), _observed(), EVENTS, rank, world, size=SIZE)
        t = R.max_over_ranks(10.0 + rank)
        np.save(out + f"/r{rank}.npy", np.concatenate([[r["ll"], t], r["g_be"], r["g_ba"], r["counts"].ravel()]))
    finally:
        td.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_covers_every_event_once():
    for n in (0, 1, 7, 64, 1001):
        for w in (1, 2, 3, 8):
            parts = [R.shard(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            assert max(h - l for l, h in parts) - min(h - l for l, h in parts) <= 1


@pytest.mark.parametrize("world", [2, 3])
def test_gradient_over_gloo_ranks_equals_one_process(world, tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    ref = R.gradient_over_ranks(_fake_gradient, _bunches(), _observed(), EVENTS, 0, 1, size=SIZE)
    for rank in range(world):
        v = np.load(tmp_path / f"r{rank}.npy")
        assert np.isclose(v[0], ref["ll"], rtol=1e-12)
        assert v[1] == 10.0 + world - 1  # the slowest rank
        assert np.allclose(v[2:2 + SIZE], ref["g_be"], rtol=1e-12)
        assert np.allclose(v[2 + SIZE:2 + 2 * SIZE], ref["g_ba"], rtol=1e-12)
        assert np.array_equal(v[2 + 2 * SIZE:].reshape(EVENTS, GSIZE), ref["counts"])
