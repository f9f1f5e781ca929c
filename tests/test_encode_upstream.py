"""mio_ce's record encoding pinned to bytes written by unmodified MERCURY6.

tests/golden/ce_upstream.npz holds the one close-encounter record of the
reference's fixture tests/fixtures/close6/upstream.ce (written by the original
MERCURY6, its README) and its header (made by
tests/golden/make_ce_upstream_golden.py). The record's fields are decoded
from the stored characters: every base-224 field that survives the record's
overlapping substring assignments (mercury6_2.for:5478-5501) at the middle of
its cell, the two 8-character fl2c fields (time and distance, whose 7-digit
mantissas resolve below one ulp) as a double that encodes to them, found by
search. States are rebuilt from the decoded mco_x2ov variables
(mercury6_2.for:3057-3086), the record is encoded again, and the 70 bytes
must be the ones MERCURY6 wrote: the oracle's restatement on the CPU, and
the library's device encoder on the GPU.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from mercuda_b200.system import K2

GOLDEN = Path(__file__).resolve().parent / "golden" / "ce_upstream.npz"
PI = 3.141592653589793
TWOPI = 2.0 * PI
EVENT = np.dtype([("i", np.int32), ("j", np.int32), ("kind", np.int32), ("now", np.int32), ("distance", np.float64),
                  ("time", np.float64), ("xi", np.float64, 6), ("xj", np.float64, 6)])


def cell(chars: bytes, lo: float, hi: float) -> float:
    """The middle of the base-224 cell the characters name, mapped to [lo, hi)."""
    idx = 0
    for c in chars:
        idx = idx * 224 + (c - 32)
    return lo + (idx + 0.5) / 224.0 ** len(chars) * (hi - lo)


def fl2c_guess(chars: bytes) -> float:
    frac = 0.0
    scale = 1.0
    for c in chars[:7]:
        scale /= 224.0
        frac += (c - 32) * scale
    return (2.0 * frac - 1.0) * 10.0 ** (chars[7] - 32 - 112)


def state(chars: bytes, rcen: float, rmax: float, mcen: float) -> np.ndarray:
    """Position and velocity whose mco_x2ov variables fall in the cells of a
    body's 24 surviving characters (fr, theta, phi, fv, vtheta, vphi: 4 each)."""
    rfac = math.log10(rmax / rcen)
    fr = cell(chars[0:4], 0.0, rfac)
    theta = cell(chars[4:8], 0.0, PI)
    phi = cell(chars[8:12], 0.0, TWOPI)
    fv = cell(chars[12:16], 0.0, 1.0)
    vtheta = cell(chars[16:20], 0.0, PI)
    vphi = cell(chars[20:24], 0.0, TWOPI)
    r = rcen * 10.0 ** fr
    temp = math.sqrt((1.0 / fv - 1.0) / 2.0)          # fv = 1 / (1 + 2 (ke / be)^2)
    v = math.sqrt(2.0 * temp * mcen / r)               # ke / be = v^2 r / (2 mcen)
    x = r * np.array([math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)])
    u = v * np.array([math.sin(vtheta) * math.cos(vphi), math.sin(vtheta) * math.sin(vphi), math.cos(vtheta)])
    return np.concatenate([x, u])


@pytest.fixture(scope="module")
def upstream():
    g = np.load(GOLDEN)
    rec = bytes(g["record"])
    mcen = round(float(g["mcen"]), 12) * K2
    rcen, rmax = round(float(g["rcen"]), 12), round(float(g["rmax"]), 12)
    ev = np.zeros(1, EVENT)
    ids = [cell(rec[8:11], 0.0, 224.0 ** 3) - 0.5, cell(rec[11:14], 0.0, 224.0 ** 3) - 0.5]
    ev["i"], ev["j"] = int(round(ids[0])) + 1, int(round(ids[1])) + 1
    ev["kind"] = 1
    ev["time"] = fl2c_guess(rec[0:8])
    ev["distance"] = fl2c_guess(rec[14:22])
    ev["xi"] = state(rec[22:46], rcen, rmax, mcen)
    ev["xj"] = state(rec[46:70], rcen, rmax, mcen)
    return rec, ev, mcen, rcen, rmax


def settle_fl2c(encode, ev, field, want: bytes, span: slice):
    """The double nearest the decoded value whose encoding gives `want` in
    the record bytes `span` (searched over +-256 ulps)."""
    x0 = float(ev[field][0])
    lo = hi = x0
    for _ in range(257):
        for x in (lo, hi):
            ev[field] = x
            if bytes(encode(ev)[0])[span] == want:
                return True
        lo = np.nextafter(lo, -np.inf)
        hi = np.nextafter(hi, np.inf)
    return False


def test_oracle_encodes_the_upstream_record(oracle, upstream):
    rec, ev, mcen, rcen, rmax = upstream
    assert (int(ev["i"][0]), int(ev["j"][0])) == (2, 3)
    enc = lambda e: oracle.mio_ce(e, mcen, rcen, rmax)
    assert settle_fl2c(enc, ev, "time", rec[0:8], slice(0, 8))
    assert settle_fl2c(enc, ev, "distance", rec[14:22], slice(14, 22))
    got = bytes(enc(ev)[0])
    assert got == rec, [k for k in range(70) if got[k] != rec[k]]


@pytest.mark.gpu
def test_device_encodes_the_upstream_record(cuda_lib, oracle, upstream):
    from mercuda_b200.backend import encode_ce
    rec, ev, mcen, rcen, rmax = upstream
    enc = lambda e: oracle.mio_ce(e, mcen, rcen, rmax)
    assert settle_fl2c(enc, ev, "time", rec[0:8], slice(0, 8))
    assert settle_fl2c(enc, ev, "distance", rec[14:22], slice(14, 22))
    got = bytes(encode_ce(ev, mcen, rcen, rmax, cuda_lib)[0])
    assert got == rec, [k for k in range(70) if got[k] != rec[k]]
