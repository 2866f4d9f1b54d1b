"""VEINSGRID_REDUCED (grids.f:1771-2073) on the device against the oracle's
sequential loops: CR01 and CONTA11 identical after the marking, for dense
sets of overlapping patches (many waves of rows), and the neighbour cap."""
import numpy as np
import pytest

from asohf_b200 import abi, api
from oracle import oracle as O

pytestmark = pytest.mark.gpu
NA = abi.NAMRX


def patch_set(nx, lado0, ir, npatch, span, seed):
    """npatch patches of level ir whose corners are cell centres of level
    ir-1 inside a cube of `span` base cells: many overlaps."""
    rng = np.random.default_rng(seed)
    dx = lado0 / nx
    dpar = dx / 2.0 ** (ir - 1)
    n3 = rng.integers(6, NA + 1, (npatch, 3)).astype(np.int32)
    base = -lado0 / 2 + 0.5 * dpar + 4 * dx
    k = rng.integers(0, int(span * 2 ** (ir - 1)), (npatch, 3))
    pr = (base + dpar * k).astype(np.float32)
    cr = np.zeros((npatch, NA, NA, NA), np.int32)
    for p in range(npatch):
        cr[p, :n3[p, 2], :n3[p, 1], :n3[p, 0]] = rng.integers(1, 50, (n3[p, 2], n3[p, 1], n3[p, 0]))
    return dx, n3, pr, cr.reshape(npatch, -1)


@pytest.mark.parametrize("ir,npatch,span,seed", [(1, 12, 8, 1), (1, 200, 24, 2), (2, 400, 16, 3), (3, 150, 6, 4)])
def test_veinsgrid_matches_oracle(gpu_lib, ir, npatch, span, seed):
    nx, lado0 = 64, 64.0
    dx, n3, pr, cr = patch_set(nx, lado0, ir, npatch, span, seed)
    radx1 = np.float32(-lado0 / 2 + 0.5 * dx)
    args = (ir, dx, float(radx1), n3[:, 0], n3[:, 1], n3[:, 2], pr[:, 0], pr[:, 1], pr[:, 2], npatch)
    cg, tg = cr.copy(), cr.copy()
    co, to = cr.copy(), cr.copy()
    api.GpuBackend().a.veinsgrid_reduced(*args, cg, tg)
    O.OracleBackend().veinsgrid_reduced(*args, co, to)
    assert np.array_equal(cg, co)
    assert np.array_equal(tg, to)
    assert (cg == 0).sum() > (cr == 0).sum()   # cells were marked


def test_veinsgrid_neighbour_cap(gpu_lib):
    dx, n3, pr, cr = patch_set(64, 64.0, 1, 40, 4, 5)   # 40 patches in 4^3 base cells: all meet
    with pytest.raises(RuntimeError):
        api.GpuBackend().a.veinsgrid_reduced(1, dx, float(-32 + 0.5 * dx), n3[:, 0], n3[:, 1], n3[:, 2], pr[:, 0],
                                             pr[:, 1], pr[:, 2], 10, cr)
