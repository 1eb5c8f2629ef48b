"""The kernel evaluates the birefringence angular functions of gpu/pro.cu:784-786 from a
table in v = sqrt(1 - |cos|) (linear interpolation, 1024 intervals).  Checked here against
the formula evaluated in double precision at random angles: the table error is below
the error of the fast-math exp/pow/atan of the reference's own GPU build (~1e-6)."""
import numpy as np

from ppc_b200.api import PPC


def test_bfr_table_matches_formula(ice_full):
    c = PPC()
    c.initialize(1.0, ice_full)
    b = np.array(list(c.params().bfr), np.float64)
    tab = np.frombuffer(c.table("bfrt"), np.float32).reshape(-1, 4)
    N = len(tab) - 1
    rng = np.random.default_rng(0)
    dot = rng.uniform(-1, 1, 200000).astype(np.float32)
    v = np.sqrt(np.maximum(0, 1 - np.abs(dot))).astype(np.float32) * np.float32(N)
    iv = np.minimum(v.astype(np.int32), N - 1)
    fv = (v - iv).astype(np.float32)
    got = tab[iv, :3] + fv[:, None] * (tab[iv + 1, :3] - tab[iv, :3])
    sdt = np.sqrt(1 - dot.astype(np.float64) ** 2)
    cdt = np.abs(dot.astype(np.float64))
    sx = np.maximum(0, b[0] * np.exp(-b[1] * np.arctan(b[3] * sdt) ** b[2]))
    sy = np.maximum(0, b[4] * np.exp(-b[5] * np.arctan(b[7] * sdt) ** b[6]))
    mx = np.maximum(0, b[8] * np.arctan(b[11] * sdt * cdt) * np.exp(-b[9] * sdt + b[10] * cdt))
    ref = np.stack([sx, sy, mx], 1)
    scale = np.abs(ref).max(axis=0)
    err = np.abs(got - ref) / scale
    assert err.max() < 4e-6, err.max(axis=0)
    c.close()
