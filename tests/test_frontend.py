"""The device front end's host side without a GPU: f2k text to source records (the TR
parsing of gpu/f2k.cxx:555-583, shared with the ppc command line)."""
import numpy as np

from ppc_b200 import types as T
from ppc_b200.api import f2k_sources

F2K = """V 2000.1
MC
TR 1 0 amu -100.0 20.0 300.0 90.0 0.0 400.0 1000.0 10.0
TR 1 0 brems -50.0 20.0 300.0 90.0 0.0 0.0 250.0 60.0
TR 1 0 hadr 0 0 0 45.0 270.0 0.0 100.0 5.0
TR 1 0 e+ 1 2 3 170.0 185.0 0.0 30.0 7.0
TR 1 0 ph 5 5 5 0 0 0 12345.7 7
TR 1 0 nu_mu 0 0 0 0 0 0 1 0
EE
"""


def _direction(th, ph):
    fcv = np.float32(np.pi) / np.float32(180)
    th = fcv * np.float32(180 - th)
    ph = fcv * np.float32(ph + 180 if ph < 180 else ph - 180)
    return np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], np.float32)


def test_f2k_text_becomes_sources():
    src, lines = f2k_sources(F2K, first_segment=10)
    assert lines == 9
    assert len(src) == 5
    assert list(src["kind"]) == [T.SRC_PARTICLE] * 4 + [T.SRC_POINT]
    assert list(src["type"][:4]) == [0, 11, 101, 13]
    assert list(src["q"]) == [12, 13, 14, 15, 16]  # one segment per line
    assert np.allclose(src["r"][0], [-100, 20, 300, 10]) and src["dr"][0] == 400 and src["amount"][0] == 1000
    assert src["amount"][4] == 12345  # "ph": an exact photon count
    for k, (th, ph) in enumerate([(90, 0), (90, 0), (45, 270), (170, 185)]):
        assert np.allclose(src["n"][k], _direction(th, ph), atol=2e-7), k
    assert np.all(src["scale"][:4] == 1)


def test_empty_and_unterminated_text():
    src, lines = f2k_sources("")
    assert len(src) == 0 and lines == 0
    src, lines = f2k_sources("TR 1 0 e- 0 0 0 0 0 0 5 0")  # no newline at the end
    assert len(src) == 1 and lines == 1 and src["type"][0] == 12 and src["q"][0] == 1
