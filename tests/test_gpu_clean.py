"""CHECK_RUBISH and ACCIDENTAL_SUBSTRUCTURE (haloes_particles.f:259-364) on
the device against the oracle's sequential loops, on random catalogues in
level order with many overlaps."""
import numpy as np
import pytest

from asohf_b200 import abi, api
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_catalogue(n, seed, zero_speed=False, nlev=4, spread=10.0, shift=0.0):
    rng = np.random.default_rng(seed)
    cat = abi.Catalogue(n + 8)
    lev = np.sort(rng.integers(0, nlev, n)).astype(np.int32)
    cat.levhal[:n] = lev
    # clustered centres so that many pairs meet the tests
    centres = rng.uniform(-spread, spread, (max(n // 20, 1), 3)) + shift
    pick = rng.integers(0, centres.shape[0], n)
    pos = centres[pick] + rng.normal(0, 0.6, (n, 3))
    cat.clusrx[:n], cat.clusry[:n], cat.clusrz[:n] = [pos[:, q].astype(np.float32) for q in range(3)]
    cat.radio[:n] = (rng.uniform(0.1, 1.5, n) / (1 + lev)).astype(np.float32)
    cat.masa[:n] = (10 ** rng.uniform(10, 13, n)).astype(np.float32)
    v = rng.normal(0, 300, (n, 3)).astype(np.float32)
    if zero_speed:
        v[rng.integers(0, n, 3)] = 0.0
    cat.vx[:n], cat.vy[:n], cat.vz[:n] = v[:, 0], v[:, 1], v[:, 2]
    cat.realclus[:n] = np.where(rng.random(n) < 0.9, -1, 0).astype(np.int32)
    cat.nclus = n
    return cat


# the last two: a wide box (the x windows prune most pairs) and centres far
# from the origin (coordinates with few bits below the radii)
CASES = [(50, 0.0, 10.0), (700, 0.0, 10.0), (3000, 0.0, 10.0), (20000, 0.0, 120.0), (3000, 4096.0, 10.0)]


@pytest.mark.parametrize("case,seed", [(c, 1 + i) for i, c in enumerate(CASES)])
def test_check_rubish_matches_oracle(gpu_lib, case, seed):
    n, shift, spread = case
    ca, cb = (random_catalogue(n, seed, shift=shift, spread=spread) for _ in range(2))
    before = int((ca.realclus[:n] == 0).sum())
    lev = ca.levhal[:n]
    for l in np.unique(lev):  # one window per level, in order, as the driver calls it
        w = np.nonzero(lev == l)[0]
        low1, low2 = int(w[0]) + 1, int(w[-1]) + 1
        kg = api.GpuBackend().check_rubish(ca, low1, low2)
        ko = O.OracleBackend().check_rubish(cb, low1, low2)
        assert kg == ko
    assert np.array_equal(ca.realclus[:n], cb.realclus[:n])
    if n >= 700:
        assert int((ca.realclus[:n] == 0).sum()) > before  # the test removes haloes


@pytest.mark.parametrize("case,seed", [(c, 11 + i) for i, c in enumerate(CASES)])
def test_accidental_substructure_matches_oracle(gpu_lib, case, seed):
    n, shift, spread = case
    ca, cb = (random_catalogue(n, seed, shift=shift, spread=spread) for _ in range(2))
    before = int((ca.realclus[:n] == 0).sum())
    kg = api.GpuBackend().accidental_substructure(ca)
    ko = O.OracleBackend().accidental_substructure(cb)
    assert kg == ko
    assert np.array_equal(ca.realclus[:n], cb.realclus[:n])
    if n >= 700:
        assert int((ca.realclus[:n] == 0).sum()) > before  # the test removes haloes


def test_zero_speed_and_level_order_are_refused(gpu_lib):
    """A zero speed leaves the Fortran's speed ratio at the previous pair's
    value: when that alone would decide a removal the call is refused, not
    guessed; so is a catalogue out of level order."""
    c = abi.Catalogue(4)
    rows = [(0, 0.0, 1.0, 1e12, 100.0), (1, 0.3, 0.5, 5e11, 0.0)]  # overlapping, the second at rest
    for i, (l, x, r, m, v) in enumerate(rows):
        c.levhal[i], c.clusrx[i], c.radio[i], c.masa[i], c.vx[i], c.realclus[i] = l, x, r, m, v, -1
    c.nclus = 2
    with pytest.raises(RuntimeError):
        api.GpuBackend().check_rubish(c, 2, 2)
    c.vx[1] = 120.0  # a regular pair: removed, no ambiguity
    assert api.GpuBackend().check_rubish(c, 2, 2) == 1
    cu = random_catalogue(300, 8)
    cu.levhal[:300] = cu.levhal[:300][::-1].copy()
    with pytest.raises(RuntimeError):
        api.GpuBackend().accidental_substructure(cu)


def test_window_edges_match_oracle(gpu_lib):
    """Pairs on the boundary of each test and a negative radius, whose reach
    is wider than the largest confirmed radius."""
    rows = [(0, 0.0, 1.0, 1e12, 100.0),
            (1, 0.5, 0.5, 5e11, 100.0),    # DIS + R = R(I) exactly: removed
            (1, -0.5, 0.5, 5e11, 100.0),   # the same on the other side
            (1, 0.75, 0.5, 5e11, 100.0),   # just outside: kept
            (1, 2.5, -2.0, 1e11, 100.0),   # 2.5 - 2 <= 1: removed
            (2, 40.0, 0.25, 1e10, 100.0),
            (2, 40.0 + 0.25 * 1.01, 0.25, 1e10, 90.0)]
    def make():
        c = abi.Catalogue(len(rows) + 2)
        for i, (l, x, r, m, v) in enumerate(rows):
            c.levhal[i], c.clusrx[i], c.radio[i], c.masa[i], c.vx[i], c.realclus[i] = l, x, r, m, v, -1
        c.nclus = len(rows)
        return c
    ca, cb = make(), make()
    assert api.GpuBackend().accidental_substructure(ca) == O.OracleBackend().accidental_substructure(cb)
    assert np.array_equal(ca.realclus[:len(rows)], cb.realclus[:len(rows)])
    assert list(cb.realclus[:5]) == [-1, 0, 0, -1, 0]
    ca, cb = make(), make()
    for low in (2, 6):
        hi = 5 if low == 2 else 7
        assert api.GpuBackend().check_rubish(ca, low, hi) == O.OracleBackend().check_rubish(cb, low, hi)
    assert np.array_equal(ca.realclus[:len(rows)], cb.realclus[:len(rows)])


def grid_catalogue(nhallev, seed, spread=10.0, sorted_levels=True):
    """Candidates as the grid finder appends them: nhallev[l] haloes of
    level l, clustered, radii shrinking with the level."""
    n = int(sum(nhallev))
    c = random_catalogue(n, seed, spread=spread)
    lev = np.repeat(np.arange(len(nhallev)), nhallev).astype(np.int32)
    if not sorted_levels:
        lev = np.random.default_rng(seed).permutation(lev).astype(np.int32)
    c.levhal[:n] = lev
    c.radio[:n] = (np.random.default_rng(seed + 100).uniform(0.2, 1.6, n) / (1 + lev)).astype(np.float32)
    return c


@pytest.mark.parametrize("nhallev,seed,spread,sorted_levels", [
    ([40, 30, 20], 1, 10.0, True),
    ([600, 500, 300, 100], 2, 10.0, True),
    ([6000, 5000, 3000, 1000], 3, 60.0, True),
    ([800, 700, 500], 4, 10.0, False),   # levels out of index order: the replay is exact anyway
])
def test_overlapping_matches_oracle(gpu_lib, nhallev, seed, spread, sorted_levels):
    ca, cb = (grid_catalogue(nhallev, seed, spread, sorted_levels) for _ in range(2))
    n = int(sum(nhallev))
    before = int((ca.realclus[:n] == 0).sum())
    for ir in range(len(nhallev)):  # as the grid finder calls it, level by level
        kg = api.GpuBackend().overlapping(ca, ir, nhallev, 0.2)
        ko = O.OracleBackend().overlapping(cb, ir, nhallev, 0.2)
        assert kg == ko
        assert np.array_equal(ca.realclus[:n], cb.realclus[:n])
    assert int((ca.realclus[:n] == 0).sum()) > before


def test_overlapping_chain_order(gpu_lib):
    """A chain of nested spheres at one point: each pair's outcome depends on
    the removals before it, in the Fortran's (I, J) order."""
    m = 64
    rows_r = np.linspace(2.0, 0.5, m).astype(np.float32)[np.random.default_rng(5).permutation(m)]
    def make():
        c = abi.Catalogue(m + 2)
        c.radio[:m] = rows_r
        c.levhal[:m] = 0
        c.realclus[:m] = -1
        c.nclus = m
        return c
    ca, cb = make(), make()
    kg = api.GpuBackend().overlapping(ca, 0, [m], 0.2)
    ko = O.OracleBackend().overlapping(cb, 0, [m], 0.2)
    assert kg == ko
    assert np.array_equal(ca.realclus[:m], cb.realclus[:m])
