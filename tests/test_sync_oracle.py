"""mxx_sync's ordering of the Small bodies (mxx_sort's Shell sort and the
furthest-first reversal, mercury6_2.for:7392-7421, 7468-7486): the library's
host routine against the oracle's restatement and, for distinct epochs,
against a plain sort; and the oracle's synchronised states against running
each prefix by hand with the oracle's mdt_bs1 steps."""
import numpy as np

from mercuda_b200.backend import epoch_order


def test_epoch_order_matches_oracle_and_sort(oracle):
    rng = np.random.default_rng(4)
    for n in (0, 1, 2, 3, 7, 40, 1000):
        e = rng.uniform(-50.0, 50.0, n)
        for tstart in (-100.0, 0.0, 100.0):
            got = epoch_order(e, tstart)
            assert np.array_equal(got, oracle.epoch_order(e, tstart))
            if n:
                want = np.argsort(e, kind="stable")
                if abs(e[want[0]] - tstart) < abs(e[want[-1]] - tstart):
                    want = want[::-1]
                assert np.array_equal(got, want)
    # ties: the library and the oracle restate the same (unstable) Shell sort
    e = np.repeat([3.0, 1.0, 2.0], 9)
    assert np.array_equal(epoch_order(e, 0.0), oracle.epoch_order(e, 0.0))


def test_oracle_sync_reaches_the_last_epoch(oracle):
    from adaptive_cases import hvar_system
    s = hvar_system(massive=False, pn=1, count=12)
    rng = np.random.default_rng(5)
    nb = s.nbig
    epochs = rng.uniform(5.0, 40.0, s.n - nb)
    order = epoch_order(epochs, 0.0)
    idx = np.concatenate([np.arange(nb), nb + order])
    s2 = s.copy()
    for name in ("m", "x", "v", "ngf", "rce", "rphys"):
        setattr(s2, name, getattr(s, name)[idx].copy())
    ep = np.concatenate([np.zeros(nb), epochs[order]])
    t, steps = oracle.mxx_sync(s2, ep, 0.0, 1.0, 1e-12, 365.25)
    assert steps > 5 and t == ep[-1]
