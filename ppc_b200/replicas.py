"""One process per GPU: sharding of events across ranks and the reductions that follow.

Photons and events are independent, so propagation needs no collective: each rank runs
its own share (the multi-GPU form of the reference's photon-range split, gpu/ppc.cu:313-320,
across processes instead of inside one).  Two things are reduced over ranks:

* device times, as the maximum (a job is as slow as its slowest rank);
* the ice gradient of a likelihood summed over events: each rank evaluates its shard of
  events and the log-likelihood, the 2 x size gradient and the per-bin charges are summed
  with one all-reduce (NCCL over NVLink for CUDA tensors, gloo on the host).
"""
import numpy as np


def shard(n, rank, world):
    """Contiguous share [lo, hi) of n items for `rank` of `world` (sizes differ by <= 1)."""
    q, r = divmod(int(n), int(world))
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def _dist():
    import torch.distributed as td
    return td if td.is_available() and td.is_initialized() else None


def _device():
    import torch
    import torch.distributed as td
    return torch.device("cuda", torch.cuda.current_device()) if td.get_backend() == "nccl" else torch.device("cpu")


def max_over_ranks(x):
    """Maximum of a float over all ranks (x itself without a process group)."""
    td = _dist()
    if td is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(a):
    """Element-wise sum of a float64 array over all ranks."""
    td = _dist()
    a = np.ascontiguousarray(a, np.float64)
    if td is None:
        return a.copy()
    import torch
    t = torch.from_numpy(a.copy()).to(_device())
    td.all_reduce(t, op=td.ReduceOp.SUM)
    return t.cpu().numpy()


def events_of_rank(bunches, events, rank, world):
    """The bunches of this rank's events (event = bunch q), renumbered from 0, and the
    rank's event range (lo, hi)."""
    lo, hi = shard(events, rank, world)
    b = bunches[(bunches["q"] >= lo) & (bunches["q"] < hi)].copy()
    b["q"] -= lo
    return b, (lo, hi)


def gradient_over_ranks(grad_fn, bunches, observed, events, rank, world, size=None, **kw):
    """Gradient of the log-likelihood summed over `events` events, the events sharded over
    ranks.  grad_fn(bunches, observed=..., events=...) is one rank's evaluation (PPC.gradient);
    observed has shape (events, gsize).  Returns the all-rank LL, g_be, g_ba and the
    (events, gsize) charges, identical on every rank."""
    b, (lo, hi) = events_of_rank(bunches, events, rank, world)
    obs = np.asarray(observed, np.float32)
    gsize = obs.shape[1]
    if hi > lo and len(b):
        r = grad_fn(b, observed=obs[lo:hi], events=hi - lo, **kw)
        ll, g_be, g_ba, counts = r["ll"], r["g_be"], r["g_ba"], r["counts"]
    else:
        if size is None:
            raise ValueError("a rank without events needs size= (ice layers)")
        ll, g_be, g_ba, counts = 0.0, np.zeros(size), np.zeros(size), np.zeros((0, gsize))
    size = len(g_be)
    full = np.zeros((events, gsize))
    full[lo:hi] = counts
    packed = np.concatenate([[ll], g_be, g_ba, full.ravel()])
    tot = sum_over_ranks(packed)
    return {"ll": float(tot[0]), "g_be": tot[1:1 + size], "g_ba": tot[1 + size:1 + 2 * size],
            "counts": tot[1 + 2 * size:].reshape(events, gsize)}
