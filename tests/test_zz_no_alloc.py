"""ppcb_propagate_noalloc: the propagation entry point that allocates no device memory.

It exists for callers that may not allocate while they run (frameworks that reserve the
GPU's memory for their own pool, steady-state loops where cudaMalloc/cudaFree would
synchronise the device).  Its scratch is a fixed static device array in the library.
Checked here through the C ABI against the existing entry point, ppcb_propagate_device,
on two calls in a row (the second must not see the first call's counters), with a list of
uneven bunches so that the offsets it computes in its scratch matter.  This file is
collected last so that a run stopping at the first failure has run every other test.
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
