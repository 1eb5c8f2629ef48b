"""ctypes / numpy mirrors of the POD records in ``ppc_b200/csrc/ppcb_types.h``.

Record layouts follow the reference data model (``gpu/ini.cxx:42-45`` DOM,
``:367-371`` hit, ``:399-419`` photon bunch, ``:431-443`` aniz/line).
"""
import ctypes as C

import numpy as np

WNUM = 512
MAXLYS = 172
LMAX = 80
LYRS = 172
CTX, CTY = 11, 10
CX, CY = 21, 19
NSTR = 240
MAXGEO = 16384
MAXRND = 131072
OMR = 0.16510
ZOFF = 1948.07


class Params(C.Structure):
    _fields_ = [
        ("size", C.c_int32), ("dh", C.c_float), ("rdh", C.c_float), ("hmin", C.c_float),
        ("ocv", C.c_float), ("sf", C.c_float), ("g", C.c_float), ("gr", C.c_float),
        ("xR", C.c_float), ("SF", C.c_float), ("G", C.c_float), ("GR", C.c_float),
        ("hr", C.c_float), ("hr2", C.c_float), ("hs", C.c_float), ("ha", C.c_float),
        ("azx", C.c_float), ("azy", C.c_float),
        ("cn", C.c_int32 * 2), ("cl", C.c_float * 2), ("crst", C.c_float * 2),
        ("cb", C.c_float * 4),
        ("tmod", C.c_int32), ("vthk", C.c_int32),
        ("lnum", C.c_int32), ("lpts", C.c_int32), ("l0", C.c_int32),
        ("lmin", C.c_float), ("lrdz", C.c_float), ("r0", C.c_float),
        ("lnx", C.c_float), ("lny", C.c_float),
        ("mmin", C.c_float * 2), ("mstp", C.c_float * 2),
        ("mnum", C.c_int32 * 2), ("mcut", C.c_int32 * 2),
        ("k1", C.c_float), ("k2", C.c_float), ("kz", C.c_float), ("fr", C.c_float),
        ("sum", C.c_float), ("bfr", C.c_float * 12), ("rx", C.c_float), ("hifl", C.c_float),
        ("gsize", C.c_int32), ("nstr", C.c_int32), ("rsize", C.c_int32), ("pad_", C.c_int32),
    ]


class Ctrl(C.Structure):
    _fields_ = [
        ("next", C.c_uint64), ("hidx", C.c_uint64), ("nan_steps", C.c_uint32),
        ("capped", C.c_uint32), ("steps", C.c_uint64), ("bad_sm", C.c_uint32 * 4),
        ("pad_", C.c_uint32 * 2),
    ]


HIT_DTYPE = np.dtype([("i", "<u4"), ("n", "<u4"), ("z", "<u4"), ("t", "<f4"),
                      ("pth", "<f4"), ("pph", "<f4"), ("dth", "<f4"), ("dph", "<f4")])

# hit accepted by the back end (ppcb_acc_hit), 56 bytes
ACC_DTYPE = np.dtype([("i", "<u4"), ("n", "<u4"), ("hit", "<u4"), ("str", "<i4"), ("om", "<i4"), ("pmt", "<i4"),
                      ("t", "<f4"), ("wv", "<f4"), ("r", "<f4", 3), ("d", "<f4", 3)])

# a light source for the device front end (ppcb_source), 72 bytes
SOURCE_DTYPE = np.dtype([("r", "<f4", 4), ("n", "<f4", 3), ("kind", "<i4"), ("amount", "<f8"), ("dr", "<f4"),
                         ("type", "<i4"), ("scale", "<f4"), ("beta", "<f4"), ("tau", "<f4"), ("fr", "<f4"),
                         ("q", "<u4"), ("pad_", "<u4")])
SRC_PARTICLE, SRC_CLST, SRC_MOPO, SRC_POINT = 0, 1, 2, 3


def source(kind, r, n=(0.0, 0.0, 1.0), amount=0.0, dr=0.0, type_=0, scale=1.0, beta=1.0, tau=0.0, fr=0.0, q=1):
    """One source record: addp (SRC_PARTICLE: amount = E [GeV], type_), addp_clst
    (SRC_CLST: amount = photons, beta), addp_mopo (SRC_MOPO: amount = light, dr = length,
    beta, tau, fr) or an f2k "ph" point (SRC_POINT: amount = photons)."""
    s = np.zeros(1, SOURCE_DTYPE)
    s["r"], s["n"], s["kind"], s["amount"], s["dr"] = r, n, kind, amount, dr
    s["type"], s["scale"], s["beta"], s["tau"], s["fr"], s["q"] = type_, scale, beta, tau, fr, q
    return s


# DirectFit likelihood records (ppcb_llh_hit / _window / _block), 24 bytes each
LLH_HIT_DTYPE = np.dtype([("str", "<i4"), ("om", "<i4"), ("t", "<f8"), ("q", "<f8")])
LLH_WINDOW_DTYPE = np.dtype([("str", "<i4"), ("om", "<i4"), ("ti", "<f8"), ("tf", "<f8")])
LLH_BLOCK_DTYPE = np.dtype([("str", "<i4"), ("om", "<i4"), ("first", "<i4"), ("last", "<i4"), ("dat", "<f8")])

# photon bunch, 64 bytes; the 16-byte union is exposed both ways
BUNCH_DTYPE = np.dtype([("r", "<f4", 4), ("n", "<f4", 4), ("q", "<u4"), ("num", "<u4"),
                        ("type", "<i4"), ("f", "<f4"), ("u", "<u4", 4)])

PBUF_DTYPE = np.dtype([("r", "<f4", 4), ("n", "<f4", 4), ("q", "<u4"), ("i", "<u4"),
                       ("fla", "<i4"), ("ofla", "<i4")])

DOM_DTYPE = np.dtype([("R", "<f4"), ("F", "<f4"), ("r", "<f4", 3)])
LINE_DTYPE = np.dtype([("n", "<i2"), ("max", "<i2"), ("x", "<f4"), ("y", "<f4"), ("r", "<f4"),
                       ("h", "<f4"), ("d", "<f4"), ("dl", "<f4"), ("dh", "<f4")])

assert HIT_DTYPE.itemsize == 32 and BUNCH_DTYPE.itemsize == 64 and PBUF_DTYPE.itemsize == 48
assert C.sizeof(Ctrl) == 56


def bunch_particle(r, n, q, num, type_, f=0.0, a=0.0, b=0.0, beta=1.0, tau=0.0, length=0.0):
    """One particle bunch (``type_`` <= 0), fields as in gpu/f2k.cxx:484-504."""
    x = np.zeros(1, BUNCH_DTYPE)
    x["r"][0] = r
    x["n"][0, :3] = n
    x["n"][0, 3] = length
    x["q"], x["num"], x["type"], x["f"] = q, num, type_, f
    x["u"][0] = np.array([a, b, beta, tau], "<f4").view("<u4")
    return x


def bunch_led(r, n, q, num, type_, ka, up, fldr, fla=-1, ofla=-1, length=0.0):
    """One LED/flasher bunch (``type_`` > 0), fields as in gpu/f2k.cxx:630-759."""
    x = np.zeros(1, BUNCH_DTYPE)
    x["r"][0] = r
    x["n"][0, :3] = n
    x["n"][0, 3] = length
    x["q"], x["num"], x["type"], x["f"] = q, num, type_, 0.0
    u = np.zeros(4, "<u4")
    u[:3] = np.array([ka, up, fldr], "<f4").view("<u4")
    u[3] = (np.uint32(np.int16(fla).view(np.uint16)) | (np.uint32(np.int16(ofla).view(np.uint16)) << 16))
    x["u"][0] = u
    return x
