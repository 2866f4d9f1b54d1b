"""asohf_re_sort_haloes (RE_SORT_HALOES, haloes_particles.f:2-56) equals
the driver's numpy restatement on random windows: drops, order, the
renumbering of REALCLUS inside the window (to 0 for a dropped target) and
outside it, NHALLEV and NCLUS, the keep mask; and nothing dropped leaves
everything as it was."""
import numpy as np
import pytest

from asohf_b200 import abi, api, driver

pytestmark = pytest.mark.gpu

FIELDS = driver.CAT_MOVE + ["realclus"]


def _cat(rng, nh, drop):
    n = int(nh.sum())
    c = abi.Catalogue(n + 8)
    c.nclus = n
    for f in driver.CAT_MOVE:
        a = getattr(c, f)
        a[:n] = (rng.integers(0, 1000, n) if a.dtype == np.int32 else rng.normal(0, 5, n)).astype(a.dtype)
    rc = rng.integers(-1, n + 1, n).astype(np.int32)   # -1, 0 and pointers in and out of the window
    rc[rng.random(n) < drop] = 0
    c.realclus[:n] = rc
    return c


@pytest.mark.parametrize("drop", [0.0, 0.3, 1.0])
def test_re_sort_matches_the_restatement(gpu_lib, drop):
    a = api.Asohf(0)
    rng = np.random.default_rng(int(drop * 10) + 1)
    for trial in range(4):
        nh = rng.integers(0, 400, 4).astype(np.int32)
        ir = int(rng.integers(0, 4))
        c1, c2 = _cat(np.random.default_rng(trial), nh, drop), _cat(np.random.default_rng(trial), nh, drop)
        if drop == 0.0:
            c1.realclus[:c1.nclus][c1.realclus[:c1.nclus] == 0] = -1
            c2.realclus[:c2.nclus][c2.realclus[:c2.nclus] == 0] = -1
        c1.nclus = c2.nclus = int(nh[:ir + 1].sum())
        n1, n2 = nh.copy(), nh.copy()
        k1 = driver.re_sort_haloes(c1, n1, ir)
        k2 = a.re_sort_haloes(c2, n2, ir)
        assert np.array_equal(n1, n2) and c1.nclus == c2.nclus
        assert np.array_equal(np.asarray(k1, bool), k2)
        m = c1.nclus
        for f in FIELDS:
            assert np.array_equal(getattr(c1, f)[:m], getattr(c2, f)[:m]), f
