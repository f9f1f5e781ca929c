"""The MVS output corrector (mco_mvs2h, mercury6_2.for:2107-2227) behind
mercury_cuda_export(h, physical=1) on the GPU, against the oracle applied to
the same downloaded state. Only the Kepler solver's cos/sin may differ from
the host's libm, so the bar is the step parity bar: 1e-12 relative with most
coordinates bit-identical."""
import numpy as np
import pytest

from mercuda_b200.backend import Backend
from mercuda_b200.system import make_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["plain", "yar", "oblate", "backwards"])
def test_export_physical_matches_oracle(cuda_lib, oracle, variant):
    sys = make_system(seed=11, n_particles=3001, nplanets=8, near_fraction=0.01, h=8.0)
    h = 8.0
    if variant == "yar":
        rng = np.random.default_rng(2)
        sys.ngf[sys.nbig:, 4] = rng.uniform(-1e-13, 1e-13, sys.n - sys.nbig)
    if variant == "oblate":
        sys.jcen[:] = [1e-6, -1e-9, 0.0]
    if variant == "backwards":
        h = -8.0
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(sys)
    for s in range(5):
        be.step(s * h, h)
    x, v = be.download()
    xe, ve = be.export(h, physical=True)
    x2, v2 = be.download()
    be.free()
    assert np.array_equal(x, x2) and np.array_equal(v, v2)  # the state is untouched
    state = sys.copy()
    state.x, state.v = x.copy(), v.copy()
    want_x, want_v = oracle.mvs_corrector(state, h, forward=True)
    assert np.all(xe[0] == 0.0)
    rx = np.max(np.abs(xe[1:] - want_x[1:]) / np.maximum(np.abs(want_x[1:]), 1e-8))
    rv = np.max(np.abs(ve[1:] - want_v[1:]) / np.maximum(np.abs(want_v[1:]), 1e-10))
    assert rx < 1e-12 and rv < 1e-12, (rx, rv)
    same = np.mean(np.all(xe == want_x, axis=1) & np.all(ve == want_v, axis=1))
    assert same > 0.9, same
    assert not np.array_equal(xe, x)


def test_export_without_physical_is_the_state(cuda_lib):
    sys = make_system(seed=3, n_particles=100, nplanets=4)
    be = Backend("MVS", cuda_lib)
    be.configure()
    be.upload(sys)
    be.step(0.0, 8.0)
    x, v = be.download()
    xe, ve = be.export(8.0, physical=False)
    be.free()
    assert np.array_equal(x, xe) and np.array_equal(v, ve)
