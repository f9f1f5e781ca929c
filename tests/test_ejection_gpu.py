"""mxx_ejec's test on the device (mercury_b200_ejections, which reads back
only the ids) against the oracle's restatement (mercury6_2.for:7071-7082) on
the positions mercury_cuda_export returns: MVS map variables (mal_hcon tests
them after mco_iden) and corrected positions, HYBRID, RADAU; the i0 = 3 form
of algorithms 11/12; an output capacity below the count; strictly beyond
rmax (a body exactly at rmax stays)."""
import ctypes as C

import numpy as np
import pytest

from adaptive_cases import hvar_system
from mercuda_b200.backend import Backend
from mercuda_b200.system import make_system, mce_init

pytestmark = pytest.mark.gpu

RADII = (0.6, 1.0, 2.5, 4.5, 5.2, 25.0, 1e4)


def test_mvs_ejections(cuda_lib, oracle):
    s = make_system(seed=4, n_particles=3001, near_fraction=0.01)
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    be.mvs_advance(0.0, 8.0, 20, 0.005)
    x, _ = be.download()
    xp, _ = be.export(8.0, physical=True)
    assert not np.array_equal(x, xp)
    seen = 0
    for rmax in RADII:
        want = oracle.mxx_ejec(x, rmax)
        assert np.array_equal(be.ejections(8.0, False, rmax), want)
        assert np.array_equal(be.ejections(8.0, True, rmax), oracle.mxx_ejec(xp, rmax))
        assert np.array_equal(be.ejections(8.0, False, rmax, i0=3), oracle.mxx_ejec(x, rmax, i0=3))
        seen += len(want)
    assert seen > 1000
    # capacity below the count: the total comes back, the first cap ids are written
    want = oracle.mxx_ejec(x, 2.5)
    ids = np.zeros(5, dtype=np.int32)
    count = C.c_int(0)
    assert cuda_lib.mercury_b200_ejections(8.0, 0, 2.5, 2, ids.ctypes.data_as(C.POINTER(C.c_int)), 5,
                                           C.byref(count)) == 0
    assert count.value == len(want) and np.array_equal(ids, want[:5])
    # a body exactly at rmax is not ejected (r^2 > rmax^2)
    j = int(want[0]) - 1
    r = float(np.sqrt(x[j] @ x[j]))
    if r * r == x[j, 0] * x[j, 0] + x[j, 1] * x[j, 1] + x[j, 2] * x[j, 2]:
        assert j + 1 not in be.ejections(8.0, False, r)
    assert cuda_lib.mercury_b200_ejections(8.0, 0, -1.0, 2, ids.ctypes.data_as(C.POINTER(C.c_int)), 5,
                                           C.byref(count)) != 0
    be.free()


@pytest.mark.parametrize("algorithm", ["HYBRID", "RADAU"])
def test_ejections_other_integrators(cuda_lib, oracle, algorithm):
    if algorithm == "HYBRID":
        s = mce_init(make_system(seed=6, n_particles=500, near_fraction=0.02), 8.0, 3.0)
    else:
        s = hvar_system(massive=True, pn=0, count=40)
    be = Backend(algorithm, cuda_lib)
    be.configure()
    be.upload(s.copy())
    x, _ = be.download()
    xp, _ = be.export(8.0, physical=True)
    assert np.array_equal(x, xp)
    for rmax in RADII:
        assert np.array_equal(be.ejections(8.0, True, rmax), oracle.mxx_ejec(x, rmax))
    be.free()
