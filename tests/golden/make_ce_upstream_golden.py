"""Extract the close-encounter record that unmodified MERCURY6 wrote into the
reference's fixture tests/fixtures/close6/upstream.ce (its README: a
Newtonian BS flyby of a particle past a 1e-12 Msun planet, central mass
1 Msun, rcen 0.005 AU, rmax 100 AU) into tests/golden/ce_upstream.npz:

    record   the 70-byte body of the '6b' line (mio_ce's c(1:70))
    header   the 62-byte header of the '6a' line (mce_init's header(1:62))
    mcen, rcen, rmax   decoded from the header (mio_fl2c fields 15:22,
                       47:54, 55:62)

Run from the repository root where the reference tree is mounted:
    python tests/golden/make_ce_upstream_golden.py <path to upstream.ce> [out.npz]
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]


def fraction(chars: bytes) -> float:
    """The base-224 digits (characters 32..255) as a fraction in [0, 1)."""
    value, scale = 0.0, 1.0
    for c in chars:
        scale /= 224.0
        value += (c - 32) * scale
    return value


def fl2c_value(chars: bytes) -> float:
    """The number mio_fl2c encoded in 8 characters (7 mantissa, 1 exponent)."""
    return (2.0 * fraction(chars[:7]) - 1.0) * 10.0 ** (chars[7] - 32 - 112)


def main(src, out):
    raw = Path(src).read_bytes()
    lines = raw.split(b"\x0c")
    head = [r for r in lines if r.startswith(b"6a")][0]
    rec = [r for r in lines if r.startswith(b"6b")][0]
    header = head[4:66]          # '6a', the algorithm as i2, then header(1:62)
    record = rec[2:72]           # '6b', then c(1:70)
    assert len(header) == 62 and len(record) == 70
    mcen = fl2c_value(header[14:22])
    rcen = fl2c_value(header[46:54])
    rmax = fl2c_value(header[54:62])
    np.savez_compressed(out, record=np.frombuffer(record, dtype=np.uint8), header=np.frombuffer(header, dtype=np.uint8),
                        mcen=np.array(mcen), rcen=np.array(rcen), rmax=np.array(rmax))
    print(f"mcen {mcen} rcen {rcen} rmax {rmax}")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2] if len(sys.argv) > 2 else ROOT / "tests/golden/ce_upstream.npz")
