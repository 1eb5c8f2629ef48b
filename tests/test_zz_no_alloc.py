"""ppcb_propagate_noalloc: the propagation entry point that allocates no device memory.

It exists for callers that may not allocate while they run (frameworks that reserve the
GPU's memory for their own pool, steady-state loops where cudaMalloc/cudaFree would
synchronise the device).  Its scratch is a fixed static device array in the library.
Checked here through the C ABI against the existing entry point, ppcb_propagate_device,
on two calls in a row (the second must not see the first call's counters), with a list of
uneven bunches so that the offsets it computes in its scratch matter; also at the largest
bunch list the scratch holds, with a hit buffer smaller than the hits produced, with no
photons, and with a photon count above the bunches' total.  This file is collected last so
that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import types as T  # noqa: E402
from ppc_b200._lib import lib  # noqa: E402
from ppc_b200.api import PPC  # noqa: E402


def _bunches(n=777, seed=3):
    rng = np.random.default_rng(seed)
    b = np.repeat(T.bunch_led([0, 0, 0, 0], [0, 0, 1], 1, 1, 1, ka=-1, up=0, fldr=-1), n)
    b["num"] = rng.integers(1, 600, n).astype(np.uint32)
    b["q"] = np.arange(n, dtype=np.uint32) + 1
    b["r"][:, 0] = rng.uniform(-60, 60, n)
    b["r"][:, 1] = rng.uniform(-60, 60, n)
    b["r"][:, 2] = rng.uniform(-300, 300, n)
    return b


def _sorted(h):
    return np.sort(h, order=["n", "i", "t", "z", "pth", "pph", "dth", "dph"])


def test_noalloc_matches_existing_entry_point_twice(ice_small):
    import torch
    c = PPC()
    c.initialize(1.0, ice_small)
    c.set_seed(21)
    c.set_options(deterministic=True)
    c.choose(0)
    c.ini()
    b = _bunches()
    num = int(b["num"].sum())
    bstart = np.concatenate([[0], np.cumsum(b["num"].astype(np.uint64))]).astype(np.uint64)
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    ds = torch.from_numpy(bstart.view(np.uint8).copy()).cuda()
    cap = 1 << 20
    dh = torch.zeros((cap, 32), dtype=torch.uint8, device="cuda")
    ctrl = torch.zeros(56, dtype=torch.uint8, device="cuda")

    # existing entry point
    c.rng_reset()
    c.propagate_device(db.data_ptr(), ds.data_ptr(), len(b), num, dh.data_ptr(), cap, ctrl.data_ptr())
    torch.cuda.synchronize()
    n_ref = T.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes()).hidx
    ref = _sorted(dh[:n_ref].cpu().numpy().view(T.HIT_DTYPE).reshape(-1))
    assert n_ref > 50

    L = lib()
    for call in range(2):
        c.rng_reset()
        dh.zero_()
        nh = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
        rc = L.ppcb_propagate_noalloc(c._c, 0, C.c_void_p(db.data_ptr()), len(b), num, C.c_void_p(dh.data_ptr()),
                                      cap, C.c_void_p(nh.data_ptr()), None)
        assert rc == 0, L.ppcb_last_error()
        torch.cuda.synchronize()
        n = int(nh.item())
        assert n == n_ref, (call, n, n_ref)
        got = _sorted(dh[:n].cpu().numpy().view(T.HIT_DTYPE).reshape(-1))
        assert np.array_equal(got, ref), call
    c.close()


def _ctx(ice, seed=21):
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(seed)
    c.set_options(deterministic=True)
    c.choose(0)
    c.ini()
    return c


def _existing(c, db, b, num, cap):
    """Hits and hit count of the existing entry point (ppcb_propagate_device)."""
    import torch
    bstart = np.concatenate([[0], np.cumsum(b["num"].astype(np.uint64))]).astype(np.uint64)
    ds = torch.from_numpy(bstart.view(np.uint8).copy()).cuda()
    dh = torch.zeros((cap, 32), dtype=torch.uint8, device="cuda")
    ctrl = torch.zeros(56, dtype=torch.uint8, device="cuda")
    c.rng_reset()
    c.propagate_device(db.data_ptr(), ds.data_ptr(), len(b), num, dh.data_ptr(), cap, ctrl.data_ptr())
    torch.cuda.synchronize()
    n = T.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes()).hidx
    return n, dh[:min(n, cap)].cpu().numpy().view(T.HIT_DTYPE).reshape(-1)


def _noalloc(c, db, nb, num, cap):
    import torch
    L = lib()
    dh = torch.zeros((max(cap, 1), 32), dtype=torch.uint8, device="cuda")
    nh = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
    c.rng_reset()
    rc = L.ppcb_propagate_noalloc(c._c, 0, C.c_void_p(db.data_ptr()), nb, num, C.c_void_p(dh.data_ptr()), cap,
                                  C.c_void_p(nh.data_ptr()), None)
    assert rc == 0, L.ppcb_last_error()
    torch.cuda.synchronize()
    n = int(nh.item())
    return n, dh[:min(n, cap)].cpu().numpy().view(T.HIT_DTYPE).reshape(-1)


def test_noalloc_at_the_largest_bunch_list(ice_small):
    """65536 bunches of uneven size (every offset of the scratch in use): the same hits as
    the existing entry point."""
    import torch
    c = _ctx(ice_small, seed=4)
    b = _bunches(n=65536, seed=9)
    b["num"] = np.random.default_rng(10).integers(1, 40, len(b)).astype(np.uint32)
    num = int(b["num"].sum())
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    n_ref, ref = _existing(c, db, b, num, 1 << 20)
    n, got = _noalloc(c, db, len(b), num, 1 << 20)
    assert n_ref > 50 and n == n_ref
    assert np.array_equal(_sorted(got), _sorted(ref))
    c.close()


def test_noalloc_hit_buffer_smaller_than_the_hits(ice_small):
    """nhits reports every hit produced; only the first hcap records are stored, and they
    are hits the full run also produces."""
    import torch
    c = _ctx(ice_small, seed=6)
    b = _bunches(seed=5)
    num = int(b["num"].sum())
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    n_ref, ref = _existing(c, db, b, num, 1 << 20)
    cap = n_ref // 3
    n, got = _noalloc(c, db, len(b), num, cap)
    assert n == n_ref and len(got) == cap
    keys = {r.tobytes() for r in ref}
    assert all(r.tobytes() in keys for r in got)
    c.close()


def test_noalloc_no_photons_and_count_above_the_total(ice_small):
    """num = 0 produces no hit; a photon count above the bunches' total is clamped to it."""
    import torch
    c = _ctx(ice_small, seed=8)
    b = _bunches(n=300, seed=7)
    num = int(b["num"].sum())
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    n0, _ = _noalloc(c, db, len(b), 0, 1024)
    assert n0 == 0
    n_ref, ref = _existing(c, db, b, num, 1 << 20)
    n, got = _noalloc(c, db, len(b), num + 5000, 1 << 20)
    assert n == n_ref and np.array_equal(_sorted(got), _sorted(ref))
    c.close()


def test_noalloc_rejects_oversized_bunch_list(ice_small):
    import torch
    c = PPC()
    c.initialize(1.0, ice_small)
    c.choose(0)
    c.ini()
    n = 65537
    b = np.repeat(T.bunch_led([0, 0, 0, 0], [0, 0, 1], 1, 1, 1, ka=-1, up=0, fldr=-1), n)
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    dh = torch.zeros((16, 32), dtype=torch.uint8, device="cuda")
    nh = torch.zeros(1, dtype=torch.int64, device="cuda")
    L = lib()
    rc = L.ppcb_propagate_noalloc(c._c, 0, C.c_void_p(db.data_ptr()), n, n, C.c_void_p(dh.data_ptr()), 16,
                                  C.c_void_p(nh.data_ptr()), None)
    assert rc == 7
    assert b"65536" in L.ppcb_last_error()
    c.close()
