"""mxx_sync's epoch synchronisation on the device (mercury_b200_sync_epochs)
against the oracle's restatement (mercury6_2.for:7442-7574 with mdt_bs1):
Small bodies at scattered epochs on either side of the Big bodies' epoch,
integrated prefix by prefix to the last epoch. mdt_bs1 on the device rounds as
the oracle's, so the common epoch, the step count and every state must be
identical."""
import numpy as np
import pytest

from adaptive_cases import hvar_system
from mercuda_b200.backend import Backend, BackendError, epoch_order

pytestmark = pytest.mark.gpu


def ordered_case(seed, lo, hi, tstart, count=60):
    s = hvar_system(massive=False, pn=1, count=count)
    rng = np.random.default_rng(seed)
    nb = s.nbig
    epochs = rng.uniform(lo, hi, s.n - nb)
    epochs[:3] = epochs[3]          # equal epochs: no step between them
    order = epoch_order(epochs, tstart)
    idx = np.concatenate([np.arange(nb), nb + order])
    for name in ("m", "x", "v", "ngf", "rce", "rphys"):
        setattr(s, name, getattr(s, name)[idx].copy())
    return s, np.concatenate([np.zeros(nb), epochs[order]])


@pytest.mark.parametrize("lo,hi,tstart", [(5.0, 40.0, 0.0), (-30.0, 25.0, -40.0)])
def test_device_sync_matches_oracle(cuda_lib, oracle, lo, hi, tstart):
    s, ep = ordered_case(7, lo, hi, tstart)
    be = Backend("BS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    t, steps = be.sync_epochs(ep, 0.0, 1.0, 1e-12, 365.25)
    x, v = be.download()
    be.free()
    ref = s.copy()
    tr, sr = oracle.mxx_sync(ref, ep, 0.0, 1.0, 1e-12, 365.25)
    assert steps > 10 and steps == sr and t == tr
    assert np.array_equal(x, ref.x) and np.array_equal(v, ref.v)


def test_sync_refuses_other_setups(cuda_lib):
    s, ep = ordered_case(8, 5.0, 40.0, 0.0, count=6)
    be = Backend("RADAU", cuda_lib)
    be.configure()
    be.upload(s.copy())
    with pytest.raises(BackendError):
        be.sync_epochs(ep, 0.0, 1.0, 1e-12, 365.25)
    be.free()
    s.m[s.nbig] = 1e-9
    be = Backend("BS", cuda_lib)
    be.configure()
    be.upload(s.copy())
    with pytest.raises(BackendError):
        be.sync_epochs(ep, 0.0, 1.0, 1e-12, 365.25)
    be.free()
