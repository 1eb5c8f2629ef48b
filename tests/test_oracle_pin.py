"""Pins the oracle (oracle/ppc_oracle.c) and the product's table build to the reference.

Two sources of truth, both the reference's own code:
  * golden vectors in tests/golden/ made by tests/golden/make_golden.py from the reference
    compiled as its CPU build (checked everywhere, no reference needed at test time);
  * the reference harness itself (oracle/_ref/ref_harness) when it was built here.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_util as O
from ppc_b200.api import PPC

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TABLES = ["az", "lr", "ls", "mcol", "sc", "lp", "absca", "wmeta", "oms", "rm", "wvs", "eff"]


def _product(ice, env, monkeypatch):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    c = PPC()
    c.initialize(1.0, ice)
    return c


@pytest.mark.parametrize("kind", ["small", "full", "full2d", "small_tilt", "small_hole", "full_ng", "small_xr1"])
def test_product_tables_match_reference_golden(kind, request):
    """The loader's table image is bit-identical to the reference's (ini::set)."""
    ice = request.getfixturevalue("ice_" + kind)
    c = PPC()
    c.initialize(1.0, ice)
    t = c.tables()
    with open(os.path.join(GOLD, f"tables_{kind}.json")) as f:
        gold = json.load(f)
    got = {k: hashlib.sha256(t[k].tobytes()).hexdigest() for k in TABLES}
    assert got == gold
    c.close()


@pytest.mark.parametrize("kind", ["full", "full2d", "small_tilt"])
def test_oracle_zshift_matches_reference_golden(kind, request):
    ice = request.getfixturevalue("ice_" + kind)
    g = np.load(os.path.join(GOLD, f"zshift_{kind}.npz"))
    c = PPC()
    c.initialize(1.0, ice)
    tb = O.tables_from_product(c)
    z = tb.zshift(g["pos"])
    assert np.array_equal(z.view(np.uint32), g["zshift"].view(np.uint32))
    c.close()


CASES = ["small_point", "full_cascade", "full2d_flasher", "small_tilt_led", "small_hole_point", "full_ng_cascade",
         "small_xr1_point"]
KIND = {"small_point": "small", "full_cascade": "full", "full2d_flasher": "full2d", "small_tilt_led": "small_tilt",
        "small_hole_point": "small_hole", "full_ng_cascade": "full_ng", "small_xr1_point": "small_xr1"}


@pytest.mark.parametrize("case", CASES)
def test_oracle_propagation_matches_reference_golden(case, request, monkeypatch):
    """Photon for photon, hit for hit: the oracle reproduces the reference's kernel-level
    hits, its phase-1 photon records and its final random-stream state."""
    g = np.load(os.path.join(GOLD, f"run_{case}.npz"))
    env = json.loads(g["env"].tobytes().decode())
    c = _product(request.getfixturevalue("ice_" + KIND[case]), env, monkeypatch)
    tb = O.tables_from_product(c)
    rm0 = int(c.tables()["rm"][0])
    seed = int(g["seed"])
    hits, pbuf, nh, s = tb.run_reference_order(g["bunch"], int(g["photons"]), 362436069 + seed, 1234567, rm0)
    assert np.array_equal(hits, g["hits"])
    assert np.array_equal(pbuf[:256], g["pbuf_head"])
    assert hashlib.sha256(pbuf.tobytes()).hexdigest().encode() == g["pbuf_sha"].tobytes()
    assert ((s.y << 32) | s.x) == int(g["rs"])
    c.close()


needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built here")


@needs_ref
@pytest.mark.parametrize("ice_name,env", [("spice_bfr-v2", {}), ("spice_ftp-v3m", {}), ("spice_bfr-v2", {"WFLA": "405"})])
def test_product_tables_match_reference_shipped_models(ice_name, env, tmp_path, monkeypatch):
    ice = os.path.join(O.REFERENCE, "ice", ice_name)
    if not os.path.isdir(ice):
        pytest.skip("reference ice models not present")
    raw = O.harness_tables(ice, tmp_path, env)
    c = _product(ice, env, monkeypatch)
    t = c.tables()
    for k in TABLES:
        assert np.frombuffer(raw[k], np.uint8).tobytes() == t[k].tobytes(), k
    c.close()


@needs_ref
@pytest.mark.parametrize("ice_name,spec,env", [
    ("spice_bfr-v2", "point:0:0:0", {"FWID": "-1", "WFLA": "405"}),
    ("spice_ftp-v3m", "flasher:63:20", {}),
    ("spice_bfr-v2", "cascade:10:20:-300:10000:0.3:0.4:0.866:11", {}),
    ("spice_ftp-v3m", "flasher:-36:30", {"FWID": "9.7"}),
])
def test_oracle_matches_reference_shipped_models(ice_name, spec, env, tmp_path, monkeypatch):
    ice = os.path.join(O.REFERENCE, "ice", ice_name)
    if not os.path.isdir(ice):
        pytest.skip("reference ice models not present")
    raw = O.harness_tables(ice, tmp_path, env)
    tb = O.tables_from_dump(raw)
    info, hits, pbuf, bunch = O.harness_run(ice, spec, 30000, 3, str(tmp_path / "r"), env)
    rm0 = int(np.frombuffer(raw["rm"], "<u4")[0])
    oh, opb, nh, s = tb.run_reference_order(bunch, 30000, 362436069 + 3, 1234567, rm0)
    assert np.array_equal(opb, pbuf)
    assert np.array_equal(oh, hits)
    assert ((s.y << 32) | s.x) == info["rs"]
