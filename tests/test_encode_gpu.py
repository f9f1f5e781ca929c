"""mio_ce's close-encounter record encoding on the device
(mercury_b200_encode_ce) against the oracle's restatement of mio_ce /
mio_fl2c / mio_re2c / mco_x2ov (mercury6_2.for:5456-5510, 5885-5918,
6926-6957, 3057-3086): the records of a fused MVS run with 2 % of the
particles near the planets, a 4,100-record burst (the size of the reference's
tests/test_events.py:19-53) and the encoder's edge cases (time 0, exact powers
of ten, negative times, ids beyond the 224^3 range, distances beyond rmax,
collision records that are not encoded)."""
import numpy as np
import pytest

from mercuda_b200.backend import EVENT_DTYPE, Backend, encode_ce
from mercuda_b200.system import K2, make_system

pytestmark = pytest.mark.gpu

RCEN, RMAX = 0.005, 100.0


def compare(cuda_lib, oracle, ev, mcen=K2):
    got = encode_ce(ev, mcen, RCEN, RMAX, cuda_lib)
    want = oracle.mio_ce(ev, mcen, RCEN, RMAX)
    assert got.shape == want.shape
    bad = np.nonzero(np.any(got != want, axis=1))[0]
    assert len(bad) == 0, (len(bad), bad[:5], bytes(got[bad[0]]), bytes(want[bad[0]]))
    return got


def test_encode_fused_run_records(cuda_lib, oracle):
    s = make_system(seed=8, n_particles=20000, near_fraction=0.02)
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(s)
    ev, _ = be.mvs_advance(0.0, 8.0, 200, RCEN)
    be.free()
    assert np.count_nonzero(ev["kind"] & 1) > 100
    lines = compare(cuda_lib, oracle, ev)
    assert lines.shape[0] == np.count_nonzero(ev["kind"] & 1)


def test_encode_burst_and_edge_cases(cuda_lib, oracle):
    rng = np.random.default_rng(3)
    n = 4100
    ev = np.zeros(n, dtype=EVENT_DTYPE)
    ev["i"] = rng.integers(1, 10, n)
    ev["j"] = rng.integers(10, 200000, n)
    ev["kind"] = 1
    ev["time"] = rng.uniform(-1e5, 1e6, n)
    ev["distance"] = np.exp(rng.uniform(np.log(1e-6), np.log(0.5), n))
    ev["xi"][:, :3] = rng.normal(0, 3, (n, 3))
    ev["xi"][:, 3:] = rng.normal(0, 0.01, (n, 3))
    ev["xj"][:, :3] = ev["xi"][:, :3] + rng.normal(0, 0.01, (n, 3))
    ev["xj"][:, 3:] = rng.normal(0, 0.01, (n, 3))
    edge = ev[:12].copy()
    edge["time"][:8] = [0.0, 1000.0, 0.001, 1.0, -10.0, 1e10, 2.5e-300, 365.25]
    edge["distance"][:4] = [1e3, 100.0, 0.1, 1e-12]
    edge["j"][8:10] = [11239424, 20000000]
    edge["kind"][10] = 2       # a collision record: not encoded
    edge["kind"][11] = 3       # both bits: encoded
    edge["xj"][11, :3] = [200.0, 0.0, 0.0]   # beyond rmax
    edge["xi"][11, :3] = [1e-4, 0.0, 0.0]    # inside rcen
    lines = compare(cuda_lib, oracle, np.concatenate([ev, edge]))
    assert lines.shape[0] == n + 11
    assert np.all(lines[n + 9, 11:14] == 255)   # an id beyond 224^3 saturates
    assert len(encode_ce(ev[:0], K2, RCEN, RMAX, cuda_lib)) == 0
