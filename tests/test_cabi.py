"""The drop-in boundary without a GPU: the C ABI loads and exports every declared entry
point; the C++ drop-in library exports the reference's xppc:: API (llh/ppc.h) so a program
written against the reference header links unchanged; errors come back as the reference's
exit statuses."""
import os
import re
import subprocess

import numpy as np
import pytest

from ppc_b200 import _lib
from ppc_b200.api import PPC, PPCError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ppc_b200", "lib")


def test_c_abi_exports_every_declared_symbol():
    L = _lib.lib()
    hdr = open(os.path.join(ROOT, "include", "ppc_b200.h")).read()
    declared = sorted(set(re.findall(r"\b(ppcb_[a-z0-9_]+)\(", hdr)))
    assert declared, "no declarations parsed"
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert set(declared) == set(_lib.EXPORTS)


XPPC_API = [
    "xppc::xrnd()", "xppc::grnd()", "xppc::start()", "xppc::stop()", "xppc::choose(int)", "xppc::ini()",
    "xppc::fin()", "xppc::eout()", "xppc::flone(unsigned long long)", "xppc::getMaxBunchSize()",
    "xppc::getWorkgroupSize()", "xppc::getTotalDeviceTime()", "xppc::initialize(float)",
    "xppc::flset(int, int)", "xppc::fldir()", "xppc::flshift(float*, float*, float*)", "xppc::set_res(float)",
    "xppc::set_res(float, float)", "xppc::efin()",
    "xppc::sett(float, float, float, std::pair<int, unsigned long long>, int, double)",
    "xppc::addp(float, float, float, float, float, float, int, float)",
    "xppc::addp_clst(float, float, float, float, unsigned long long, float, float)",
    "xppc::addp_mopo(float, float, float, float, float, float, float, float, float)",
    "xppc::hitz", "xppc::i3oms", "xppc::omts", "xppc::hvs", "xppc::rdes", "xppc::nextgen",
]


def test_xppc_library_exports_reference_api():
    out = subprocess.run(["nm", "-DC", "--defined-only", os.path.join(LIB, "libxppc.so")], capture_output=True,
                         text=True, check=True).stdout
    missing = [s for s in XPPC_API if s not in out]
    assert not missing, missing


LLH_LIKE = r"""
#include <cmath>
#include <map>
#include <vector>
#include <cstdio>
#include HEADER
int main(int argc, char** argv) {
  if (argc < 2) return 0;            // linked, not run: needs a GPU
  xppc::start();
  xppc::initialize(1.f);
  xppc::choose(-1);
  xppc::ini();
  xppc::flset(63, 20);
  xppc::sett(0, 0, 1, std::make_pair(1, 2ULL), 0);
  xppc::flone(1000000);
  xppc::eout();
  for (xppc::outz::const_iterator i = xppc::hitz.begin(); i != xppc::hitz.end(); ++i)
    printf("%d %d %zu\n", i->first.omkey.str, i->first.omkey.dom, i->second.size());
  xppc::efin();
  xppc::fin();
  xppc::stop();
  printf("%zu %zu %g %f\n", xppc::getMaxBunchSize(), xppc::getWorkgroupSize(), xppc::getTotalDeviceTime(), xppc::xrnd());
  return 0;
}
"""


@pytest.mark.parametrize("header", ["ours", "reference"])
def test_program_written_against_api_links(header, tmp_path):
    if header == "reference":
        import oracle_util as O
        h = os.path.join(O.REFERENCE, "llh", "ppc.h")
        if not O.REFERENCE or not os.path.exists(h):
            pytest.skip("reference header not present")
        src = LLH_LIKE.replace("HEADER", '"' + h + '"')
    else:
        src = LLH_LIKE.replace("HEADER", '"' + os.path.join(ROOT, "include", "xppc.h") + '"')
    f = tmp_path / "llh_like.cxx"
    f.write_text(src)
    exe = tmp_path / "llh_like"
    r = subprocess.run(["/usr/bin/g++", "-O1", "-std=c++11", str(f), "-o", str(exe), "-L" + LIB, "-lxppc",
                        "-Wl,-rpath," + LIB, "-Wl,--no-undefined"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert subprocess.run([str(exe)]).returncode == 0


def test_missing_configuration_reports_reference_status(tmp_path):
    c = PPC()
    with pytest.raises(PPCError) as e:
        c.initialize(1.0, str(tmp_path / "nowhere"))
    assert e.value.code == 1 and "cfg.txt" in str(e.value)
    c.close()


def test_corrupt_ice_table_is_rejected(tmp_path, ice_small):
    import shutil
    d = tmp_path / "ice"
    shutil.copytree(ice_small, d)
    lines = (d / "icemodel.dat").read_text().splitlines()
    lines[5] = lines[5].split()[0] + " -1 0.01 0"  # negative scattering
    (d / "icemodel.dat").write_text("\n".join(lines) + "\n")
    c = PPC()
    with pytest.raises(PPCError) as e:
        c.initialize(1.0, str(d))
    assert e.value.code == 1 and "Invalid value of ice parameter" in str(e.value)
    c.close()


def test_ice_coefficients_round_trip_and_reject_bad_values(ice_small):
    """ppcb_get_ice / ppcb_set_ice on the host table (no device needed before ini)."""
    rows = np.loadtxt(os.path.join(ice_small, "icemodel.dat"))
    c = PPC()
    c.initialize(1.0, ice_small)
    be, ba = c.get_ice()
    assert np.allclose(be, rows[:, 1].astype(np.float32)) and np.allclose(ba, rows[:, 2].astype(np.float32))
    before = c.table("absca")
    c.set_ice(be * 1.5, None)
    be2, ba2 = c.get_ice()
    assert np.allclose(be2, be * 1.5) and np.array_equal(ba2, ba)
    assert c.table("absca") != before
    bad = ba.copy()
    bad[3] = -1.0
    with pytest.raises(PPCError) as e:
        c.set_ice(None, bad)
    assert "Invalid value of ice parameter" in str(e.value)
    assert np.array_equal(c.get_ice()[1], ba)  # restored
    c.set_options(photon_streams=True)
    assert _lib.lib().ppcb_set_options(c._c, 3, 0, 0) == 7  # PPCB_EARG
    c.close()


def test_propagation_before_ini_is_an_error(ice_small):
    c = PPC()
    c.initialize(1.0, ice_small)
    from ppc_b200 import types as T
    b = T.bunch_led([0, 0, 0, 0], [0, 0, 1], 1, 10, 1, ka=-1, up=0, fldr=-1)
    with pytest.raises(PPCError) as e:
        c.propagate(b)
    assert e.value.code == 6
    c.close()


def test_result_array_must_be_hit_records(ice_small):
    """PPC.propagate(out=...) takes only a contiguous array of hit records (checked before
    any work is done)."""
    import numpy as np
    from ppc_b200 import types as T
    c = PPC()
    c.initialize(1.0, ice_small)
    b = T.bunch_led([0, 0, 0, 0], [0, 0, 1], 1, 10, 1, ka=-1, up=0, fldr=-1)
    for bad in (np.zeros(10, np.float32), np.zeros(20, T.HIT_DTYPE)[::2]):
        with pytest.raises(TypeError):
            c.propagate(b, out=bad)
    c.close()


def test_flasher_setup_matches_reference_semantics(ice_full, monkeypatch):
    """flset/fldir/flshift are host-side (gpu/f2k.cxx:590-765)."""
    monkeypatch.setenv("FLDR", "30")
    c = PPC()
    c.initialize(1.0, ice_full)
    d = c.flset(40, 30)
    assert d["r"][2] > -600 and d["r"][2] < 600
    n = c.fldir()
    up = np.float32(-0.2) * np.float32(np.pi / 180)
    assert abs(n[2] - np.sin(up)) < 1e-6
    assert abs(np.arctan2(n[1], n[0]) - np.radians(30)) < 1e-5
    # flshift: rotating the vertical frame onto itself is the identity
    out = c.flshift([0, 0, 1], [0.6, 0.0, 0.8])
    assert np.allclose(out, [0.6, 0.0, 0.8])
    out = c.flshift([1, 0, 0], [0.0, 0.0, 1.0])
    assert np.allclose(out, [1.0, 0.0, 0.0], atol=1e-6)
    c.close()


def test_gradient_checks_charge_bin_sizes(ice_small):
    """PPC.gradient rejects observed/weights arrays whose size is not the number of charge
    bins (gsize, or events x gsize) before anything reaches the device."""
    from ppc_b200 import types as T
    c = PPC()
    c.initialize(1.0, ice_small)
    gs = c.info()["gsize"]
    b = T.bunch_led([0, 0, 0, 0], [0, 0, 1], 0, 10, 1, ka=-1, up=0, fldr=-1)
    with pytest.raises(ValueError):
        c.gradient(b, weights=np.zeros(gs + 1, np.float32))
    with pytest.raises(ValueError):
        c.gradient(b, observed=np.zeros(gs, np.float32), events=3)
    with pytest.raises(PPCError) as e:  # right sizes, but no ini(): the library refuses
        c.gradient(b, weights=np.zeros((3, gs), np.float32), events=3)
    assert e.value.code == 6
    c.close()


def test_record_layouts_match_the_c_header(tmp_path):
    """Every record the Python side exchanges with the C ABI has the C compiler's size and
    field offsets (a mismatch makes a copy-out call overrun the Python buffer)."""
    from ppc_b200 import types as T
    src = tmp_path / "sz.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "ppc_b200.h"
#define F(t, m) printf(#t "." #m " %zu\\n", offsetof(t, m))
int main(void) {
  printf("ppcb_hitz_rec %zu\\n", sizeof(ppcb_hitz_rec));
  printf("ppcb_hit %zu\\n", sizeof(ppcb_hit));
  printf("ppcb_bunch %zu\\n", sizeof(ppcb_bunch));
  printf("ppcb_run_info %zu\\n", sizeof(ppcb_run_info));
  printf("ppcb_info %zu\\n", sizeof(ppcb_info));
  printf("ppcb_batch_info %zu\\n", sizeof(ppcb_batch_info));
  printf("ppcb_tune_info %zu\\n", sizeof(ppcb_tune_info));
  printf("ppcb_grad_info %zu\\n", sizeof(ppcb_grad_info));
  printf("ppcb_ctrl %zu\\n", sizeof(ppcb_ctrl));
  printf("ppcb_params %zu\\n", sizeof(ppcb_params));
  printf("ppcb_acc_hit %zu\\n", sizeof(ppcb_acc_hit));
  printf("ppcb_llh_hit %zu\\n", sizeof(ppcb_llh_hit));
  printf("ppcb_source %zu\\n", sizeof(ppcb_source));
  printf("ppcb_llh_window %zu\\n", sizeof(ppcb_llh_window));
  printf("ppcb_llh_block %zu\\n", sizeof(ppcb_llh_block));
  printf("ppcb_llh_opts %zu\\n", sizeof(ppcb_llh_opts));
  printf("ppcb_llh_info %zu\\n", sizeof(ppcb_llh_info));
  F(ppcb_hitz_rec, t0); F(ppcb_hitz_rec, str); F(ppcb_hitz_rec, r); F(ppcb_hitz_rec, n);
  return 0;
}
""")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    c = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                      check=True).stdout.splitlines())
    import ctypes as C
    py = {"ppcb_hitz_rec": _lib.HITZ_DTYPE.itemsize, "ppcb_hit": T.HIT_DTYPE.itemsize,
          "ppcb_bunch": T.BUNCH_DTYPE.itemsize, "ppcb_run_info": C.sizeof(_lib.RunInfo),
          "ppcb_info": C.sizeof(_lib.Info), "ppcb_batch_info": C.sizeof(_lib.BatchInfo),
          "ppcb_tune_info": C.sizeof(_lib.TuneInfo), "ppcb_grad_info": C.sizeof(_lib.GradInfo),
          "ppcb_ctrl": C.sizeof(T.Ctrl), "ppcb_params": C.sizeof(T.Params), "ppcb_acc_hit": T.ACC_DTYPE.itemsize,
          "ppcb_llh_hit": T.LLH_HIT_DTYPE.itemsize, "ppcb_source": T.SOURCE_DTYPE.itemsize, "ppcb_llh_window": T.LLH_WINDOW_DTYPE.itemsize,
          "ppcb_llh_block": T.LLH_BLOCK_DTYPE.itemsize, "ppcb_llh_opts": C.sizeof(_lib.LlhOpts),
          "ppcb_llh_info": C.sizeof(_lib.LlhInfo)}
    for k, v in py.items():
        assert int(c[k]) == v, (k, c[k], v)
    d = _lib.HITZ_DTYPE
    for f in ("t0", "str", "r", "n"):
        assert int(c[f"ppcb_hitz_rec.{f}"]) == d.fields[f][1], f
