"""COMPUTE_EPOT's sampling branch (haloes_particles.f:1568-1626) in the
oracle: the same seed gives the same catalogue, another seed a different
estimate, and the estimate agrees with the direct pair sum within its
sampling error.  The reference seeds RANDOM_NUMBER with an unseeded
RANDOM_SEED(), so its own estimate changes from run to run; the library and
the oracle draw from a seeded counter-based generator instead."""
import ctypes as C

import numpy as np

from asohf_b200 import driver, synth
from oracle import oracle as O


def _run(max_part_dsum, seed=1):
    s = synth.generate("small")
    plan = driver.prepare(s)
    plan.consts.do_compute_energies = 1
    plan.consts.max_part_dsum = max_part_dsum
    O.lib().orc_set_epot_seed(C.c_uint32(seed))
    try:
        r = driver.execute(plan, O.OracleBackend(), with_subs=True)
    finally:
        O.lib().orc_set_epot_seed(C.c_uint32(1))
    return r


def test_sampling_estimate_tracks_the_direct_sum():
    lim = 150
    direct = _run(10 ** 9)
    sampled = _run(lim)
    n = direct.cat.nclus
    live = direct.cat.realclus[:n] != 0
    assert np.array_equal(sampled.cat.realclus[:n], direct.cat.realclus[:n])
    big = live & (direct.cat.dmpclus[:n] >= lim)
    assert big.sum() >= 5
    a = sampled.cat.potential_e[:n][big].astype(np.float64)
    b = direct.cat.potential_e[:n][big].astype(np.float64)
    assert (a < 0).all() and (b < 0).all()
    rel = np.abs(a / b - 1.0)
    # NSAMPLE^2 >= 107^2 pairs per halo: a few per cent of sampling error
    assert np.median(rel) < 0.1, rel
    assert rel.max() < 0.5, rel
    # below the limit the direct sum is kept
    small = live & (direct.cat.dmpclus[:n] < lim)
    assert np.array_equal(sampled.cat.potential_e[:n][small], direct.cat.potential_e[:n][small])


def test_sampling_is_reproducible_and_seeded():
    a, b, c = _run(150, 1), _run(150, 1), _run(150, 7)
    n = a.cat.nclus
    big = (a.cat.realclus[:n] != 0) & (a.cat.dmpclus[:n] >= 150)
    assert np.array_equal(a.cat.potential_e[:n], b.cat.potential_e[:n])
    assert np.array_equal(a.cat.iplip[:n], b.cat.iplip[:n])
    assert not np.array_equal(a.cat.potential_e[:n][big], c.cat.potential_e[:n][big])
