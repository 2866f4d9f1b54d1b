"""Known answers of the oracle's CHECK_RUBISH and ACCIDENTAL_SUBSTRUCTURE
(haloes_particles.f:259-364) on hand-built catalogues."""
import numpy as np

from asohf_b200 import abi
from oracle import oracle as O


def cat_of(rows):
    """rows: (level, x, y, z, radius, mass, speed, realclus)"""
    c = abi.Catalogue(len(rows) + 2)
    for i, (l, x, y, z, r, m, v, rc) in enumerate(rows):
        c.levhal[i], c.clusrx[i], c.clusry[i], c.clusrz[i] = l, x, y, z
        c.radio[i], c.masa[i], c.vx[i], c.realclus[i] = r, m, v, rc
    c.nclus = len(rows)
    return c


def test_check_rubish_known_answers():
    rows = [(0, 0.0, 0.0, 0.0, 1.0, 1e12, 100.0, -1),   # host
            (1, 0.5, 0.0, 0.0, 0.6, 5e11, 120.0, -1),   # inside 1.01*0.6, mass ratio 0.5: removed
            (1, 0.5, 0.0, 0.0, 0.6, 1e11, 120.0, -1),   # mass ratio 0.1: kept
            (1, 3.0, 0.0, 0.0, 0.6, 5e11, 120.0, -1),   # too far: kept
            (1, 0.2, 0.0, 0.0, 0.6, 5e11, 500.0, -1)]   # |dv|/v = 0.8 < 3: removed
    c = cat_of(rows)
    k = O.OracleBackend().check_rubish(c, 2, 5)
    assert k == 2
    assert list(c.realclus[:5]) == [-1, 0, -1, -1, 0]


def test_accidental_substructure_known_answers():
    rows = [(0, 0.0, 0.0, 0.0, 1.0, 1e12, 100.0, -1),
            (1, 0.3, 0.0, 0.0, 0.5, 1e11, 100.0, -1),   # 0.3 + 0.5 <= 1: removed
            (1, 0.6, 0.0, 0.0, 0.5, 1e11, 100.0, -1),   # 1.1 > 1: kept
            (2, 0.6, 0.0, 0.0, 0.3, 1e10, 100.0, -1)]   # inside the kept level-1 halo: removed
    c = cat_of(rows)
    k = O.OracleBackend().accidental_substructure(c)
    assert k == 2
    assert list(c.realclus[:4]) == [-1, 0, -1, 0]


def test_overlapping_known_answers():
    """OVERLAPPING (haloes_grids.f:27-201) at level 1 of a two-level list."""
    rows = [(0, 0.0, 0.0, 0.0, 1.0, 1e12, 100.0, -1),   # level 0
            (0, 5.0, 0.0, 0.0, 1.0, 1e12, 100.0, -1),   # level 0
            (1, 0.2, 0.0, 0.0, 0.5, 1e11, 100.0, -1),   # nested in halo 1 (|1-0.5| >= 0.2): removed
            (1, 6.1, 0.0, 0.0, 1.0, 1e11, 100.0, -1),   # equal radii 1.1 apart: lens 0.26 of a sphere
            (1, 9.0, 0.0, 0.0, 0.3, 1e11, 100.0, -1),   # alone: kept
            (1, 9.0, 0.0, 0.1, 2.0, 1e11, 100.0, -1)]   # contains the one before, larger, same level:
                                                         # the smaller (row 5) is removed
    c = cat_of(rows)
    k = O.OracleBackend().overlapping(c, 1, [2, 4], 0.2)
    assert list(c.realclus[:6]) == [-1, -1, 0, 0, 0, -1]
    assert k == 3
    c = cat_of(rows)
    O.OracleBackend().overlapping(c, 1, [2, 4], 0.3)   # above the lens fraction: row 4 kept
    assert list(c.realclus[:6]) == [-1, -1, 0, -1, 0, -1]


def test_overlapping_row_flag_read_once():
    """OVERLAPPING reads the row halo's REALCLUS once per row (BASINT,
    haloes_grids.f:106-107): a row halo removed by its first partner still
    removes its later partners."""
    rows = [(0, 0.0, 0.0, 0.0, 1.0, 1e12, 100.0, -1),   # I: radius 1
            (0, 0.1, 0.0, 0.0, 3.0, 1e12, 100.0, -1),   # contains I, larger, same level: I removed
            (0, -0.2, 0.0, 0.0, 0.3, 1e12, 100.0, -1)]  # inside I: removed by I although I is gone
    c = cat_of(rows)
    O.OracleBackend().overlapping(c, 0, [3], 0.2)
    assert list(c.realclus[:3]) == [0, -1, 0]
