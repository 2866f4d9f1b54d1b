"""CREATE_MESH particle counts (grids.f:94-143 base grid, grids.f:341-380
patches) on the device against the oracle's loops: bit-exact int32 grids,
species weights, clamping of particles outside the box, border zeroing."""
from types import SimpleNamespace

import numpy as np
import pytest

from asohf_b200 import abi, api
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def particles(n, lado0, seed, outside=0.01):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-0.4 * lado0, 0.4 * lado0, (16, 3))
    pos = centres[rng.integers(0, 16, n)] + rng.normal(0, 0.03 * lado0, (n, 3))
    far = rng.random(n) < outside  # a few beyond the faces: clamped to the edge cells
    pos[far] = rng.uniform(-0.7 * lado0, 0.7 * lado0, (int(far.sum()), 3))
    pos = pos.astype(np.float32)
    z = np.zeros(n, np.float32)
    return SimpleNamespace(x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), vx=z, vy=z, vz=z,
                           m=np.ones(n, np.float32), id=np.arange(1, n + 1, dtype=np.int32))


def backends(parts):
    g, o = api.GpuBackend(), O.OracleBackend()
    g.upload(parts)
    o.upload(parts)
    return g, o


@pytest.mark.parametrize("nx,n,bor,esp", [(32, 20000, 1, [15000, 4000, 1000]),
                                           (64, 200000, 2, [200000]),
                                           (48, 50000, 0, [30000, 10000])])  # last: 10000 past the ranges
def test_base_counts_match_oracle(gpu_lib, nx, n, bor, esp):
    lado0 = 40.0
    dx = lado0 / nx
    g, o = backends(particles(n, lado0, nx))
    cg = g.a.mesh_base_counts(nx, dx, 8, bor, esp)
    co = o.mesh_base_counts(nx, dx, 8, bor, esp)
    assert np.array_equal(cg, co)
    assert cg.max() > 8


def random_patches(nx, lado0, irpa, npatch, seed):
    rng = np.random.default_rng(seed)
    dx = lado0 / nx
    radx = -lado0 / 2 + dx * (np.arange(nx + 2, dtype=np.float32) - 0.5)  # base cell centres RADX(0..NX+1)
    n3 = rng.integers(4, abi.NAMRX + 1, (npatch, 3)).astype(np.int32)
    corner = rng.integers(1, nx - abi.NAMRX // 2, (npatch, 3))
    # a level-irpa patch starts at a cell centre of its parent level
    dpar = dx / 2.0 ** (irpa - 1)
    pr = np.stack([radx[corner[:, a]] + dpar * rng.integers(0, 4, npatch) for a in range(3)], 1)
    return n3, pr.astype(np.float32)


@pytest.mark.parametrize("irpa,npatch,boramr,esp", [(1, 40, 1, [15000, 4000, 1000]),
                                                     (2, 120, 2, [10000, 5000, 5000]),
                                                     (3, 60, 0, [20000])])
def test_patch_counts_match_oracle(gpu_lib, irpa, npatch, boramr, esp):
    nx, lado0, n = 32, 40.0, 20000
    dx = lado0 / nx
    g, o = backends(particles(n, lado0, 7 + irpa, outside=0.0))
    n3, pr = random_patches(nx, lado0, irpa, npatch, irpa)
    args = (n3[:, 0], n3[:, 1], n3[:, 2], pr[:, 0], pr[:, 1], pr[:, 2])
    cg = g.a.mesh_patch_counts(nx, lado0, dx, irpa, 8, boramr, esp, *args)
    co = o.mesh_patch_counts(irpa, dx, 8, boramr, esp, *args)
    assert np.array_equal(cg, co)
    assert (cg > 0).sum() > 100
