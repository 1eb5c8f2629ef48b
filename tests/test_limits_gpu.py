"""The kernel's own limits made to fire, through the C ABI:

  * the per-photon step cap (ppcb_set_options max_steps; counted in the control block's
    `capped` and reported by ppcb_propagate's run info), a safety limit the reference does
    not have;
  * the guard on a non-finite optical depth (gpu/pro.cu:728, reported at gpu/ppc.cu:262-265):
    the step is counted in `nan_steps`, the SM it ran on recorded, and the photon dropped.

Both are driven by ordinary inputs (a small cap; a bunch whose direction is NaN, which
makes the absorption depth NaN on the photon's first step); every table index the kernel
computes stays in range for them (NaN converts to index 0 and is clamped)."""
import numpy as np
import pytest

from conftest import have_gpu

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_gpu(), reason="needs a CUDA GPU")]

from ppc_b200 import types as T  # noqa: E402
from ppc_b200.api import PPC  # noqa: E402


def _ctx(ice, **opts):
    c = PPC()
    c.initialize(1.0, ice)
    c.set_seed(31)
    c.set_options(**opts)
    c.choose(0)
    c.ini()
    return c


def _iso(num):
    return T.bunch_led([0, 0, 0, 0], [0, 0, 1], 1, num, 1, ka=-1, up=0, fldr=-1)


def test_step_cap_stops_photons_and_is_reported(ice_small):
    num = 100_000
    c = _ctx(ice_small)
    _, free = c.propagate(_iso(num))
    assert free["capped"] == 0 and free["steps"] > 10 * num  # tens of steps per photon uncapped
    c.close()

    c = _ctx(ice_small, max_steps=3)
    hits, info = c.propagate(_iso(num))
    assert info["photons"] == num
    # most photons live longer than three steps: those are stopped after exactly three, the
    # others ended (absorbed, or on a DOM) before the cap
    assert num // 2 < info["capped"] <= num, info
    assert 3 * info["capped"] <= info["steps"] <= 3 * num, info

    # the same through the device entry point: the count is in the caller's control block
    import torch
    b = _iso(num)
    db = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    ds = torch.tensor([0, num], dtype=torch.int64, device="cuda")
    dh = torch.zeros((1 << 16, 32), dtype=torch.uint8, device="cuda")
    ctrl = torch.zeros(56, dtype=torch.uint8, device="cuda")
    c.propagate_device(db.data_ptr(), ds.data_ptr(), 1, num, dh.data_ptr(), 1 << 16, ctrl.data_ptr())
    torch.cuda.synchronize()
    cc = T.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes())
    assert num // 2 < cc.capped <= num and 3 * cc.capped <= cc.steps <= 3 * num
    c.close()


def test_non_finite_direction_is_counted_and_dropped(ice_small):
    nbad, ngood = 5000, 200_000
    a = 2.01849 + 0.63176 * np.log(1e4)
    b = 0.39652 * 0.910 / 0.9216 / 0.63207
    nan = float("nan")
    bad = T.bunch_particle([0, 0, 0, 0], [nan, nan, nan], 1, nbad, -11, f=0.0, a=a, b=b)
    good = _iso(ngood)
    good["q"] = 2
    c = _ctx(ice_small)
    hits, info = c.propagate(np.concatenate([bad, good]))
    # every photon of the NaN bunch ends on its first step, counted once; the rest propagate
    assert info["nan_steps"] == nbad, info
    assert info["photons"] == nbad + ngood
    assert len(hits) > 100 and set(np.unique(hits["n"])) == {2}
    assert np.all(np.isfinite(hits["t"]))

    # device entry point: the count and the SMs of the first such steps in the control block
    import torch
    db = torch.from_numpy(bad.view(np.uint8).copy()).cuda()
    ds = torch.tensor([0, nbad], dtype=torch.int64, device="cuda")
    dh = torch.zeros((1024, 32), dtype=torch.uint8, device="cuda")
    ctrl = torch.zeros(56, dtype=torch.uint8, device="cuda")
    c.propagate_device(db.data_ptr(), ds.data_ptr(), 1, nbad, dh.data_ptr(), 1024, ctrl.data_ptr())
    torch.cuda.synchronize()
    cc = T.Ctrl.from_buffer_copy(ctrl.cpu().numpy().tobytes())
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    assert cc.nan_steps == nbad and cc.hidx == 0 and cc.steps == nbad
    assert all(0 <= s < sms for s in cc.bad_sm)
    c.close()
