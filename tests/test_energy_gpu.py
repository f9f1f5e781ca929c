"""mercury_b200_energy (mxx_en on the device) against the oracle's mxx_en of
the exported state, bit for bit: MVS with and without the output corrector,
oblateness, spins; HYBRID with its democratic-heliocentric velocity shift and
massive Small bodies in the massive set; RADAU with massive Small bodies
between massless ones."""
import numpy as np
import pytest

from adaptive_cases import hvar_system
from mercuda_b200.backend import Backend
from mercuda_b200.system import K2, make_system, mce_init

pytestmark = pytest.mark.gpu


def check(be, oracle, sys0, h, physical, spin=None):
    x, v = be.export(h, physical)
    want = oracle.mxx_en(sys0.m, x, v, sys0.jcen, spin)
    got = be.energy(h, physical, spin)
    assert got == want, (got, want)
    return got


@pytest.mark.parametrize("physical", [0, 1])
def test_mvs_energy_matches_oracle(cuda_lib, oracle, physical):
    s = make_system(seed=3, n_particles=3000, near_fraction=0.01)
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    e0 = check(be, oracle, s, 8.0, physical)
    be.mvs_advance(0.0, 8.0, 46, 0.005)
    e1 = check(be, oracle, s, 8.0, physical)
    be.free()
    # the planets' energy is conserved to the MVS map's level over a year
    assert abs(e1[0] - e0[0]) <= 1e-5 * abs(e0[0])


def test_mvs_oblateness_and_spin(cuda_lib, oracle):
    """Oblateness terms and the spin sum (every body's spin, in body order)."""
    s = make_system(seed=8, n_particles=600)
    rng = np.random.default_rng(8)
    s.jcen[:] = [1e-8, -3e-13, 2e-17]
    spin = rng.normal(size=(s.n, 3)) * 1e-12
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    be.mvs_advance(0.0, 8.0, 31, 0.005)
    for physical in (0, 1):
        check(be, oracle, s, 8.0, physical, spin)
    be.free()


def test_hybrid_energy_matches_oracle(cuda_lib, oracle):
    s = mce_init(make_system(seed=5, n_particles=800), 8.0, 3.0)
    idx = s.nbig + np.arange(5)
    s.m[idx] = 1e-11 * K2   # massive Small bodies: the massive set holds them
    be = Backend("HYBRID", cuda_lib)
    be.configure()
    work = s.copy()
    be.upload(work)
    state = {"dtflag": 0}
    t = 0.0
    for _ in range(6):
        be.hybrid_step(work, t, 8.0, 1e-12, state, 0.005)
        t += 8.0
    for physical in (0, 1):
        check(be, oracle, s, 8.0, physical)
    be.free()


def test_radau_energy_matches_oracle(cuda_lib, oracle):
    s = hvar_system(massive=True, pn=True)
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(s.copy())
    h, dtflag, t = 2.0, 0, 0.0
    for _ in range(5):
        hdid, h = be.step(t, h, 1e-12, dtflag)
        dtflag = 2
        t += hdid
    check(be, oracle, s, h, 1)
    be.free()
