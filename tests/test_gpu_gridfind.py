"""HALOFIND_GRID at the base level (haloes_grids.f:287-582) on the device
against the oracle: the candidate peaks, their order, the shell growth, the
keep/skip of covered peaks and OVERLAPPING.  The device adds the shell sums
in the Fortran's order, so the catalogue must be identical: halo count,
centres, radii, masses and the centre-of-mass columns (including the
reference's restart of BASX..BASZ from the box bound every shell).

Inputs: top-hat overdensities (two haloes of known radius), and the density
contrast of the synthetic snapshots (DENSITY + RENORM_DENSITY on the base
grid: 32^3 and 64^3 particles, and the 512^3 benchmark recipe at 1/64 of the
volume on a 128^3 grid), with the parameters of the golden vectors
(CONTRASTEC = 200, unit background factors) and with the snapshot's own
cosmology."""
import numpy as np
import pytest

from asohf_b200 import abi, api, driver, grid, synth
from oracle import oracle as O
from tests.test_oracle_kat import _tophat_field

pytestmark = pytest.mark.gpu

COLS_I = ["realclus", "levhal", "patchclus"]
COLS_F = ["clusrx", "clusry", "clusrz", "radio", "masa", "clusrxcm", "clusrycm", "clusrzcm"]


def _both(nx, dx, u, radx, args, cap=200000):
    cg, co = abi.Catalogue(cap), abi.Catalogue(cap)
    ng = api.GpuBackend().halofind_grid_base(nx, dx, u, radx, *args, cg)
    no = O.OracleBackend().halofind_grid_base(nx, dx, u, radx, *args, co)
    return ng, cg, no, co


def _same(ng, cg, no, co):
    assert ng == no and cg.nclus == co.nclus
    n = co.nclus
    for f in COLS_I + COLS_F:
        a, b = getattr(cg, f)[:n], getattr(co, f)[:n]
        assert np.array_equal(a, b, equal_nan=True), (f, np.nonzero(a != b)[0][:10])


def test_tophat_haloes(gpu_lib):
    nx, lado0 = 48, 48.0
    radx, dx = grid.malla(nx, lado0)
    u = _tophat_field(nx, [((12, 14, 20), 3.0, 400.0), ((34, 30, 26), 4.0, 300.0), ((20, 30, 10), 2.0, 600.0)])
    ng, cg, no, co = _both(nx, float(dx), u, radx, (200.0, 1.0, 1.0, 1.0, 1.0, 10.0, 0.2))
    assert ng == 3
    _same(ng, cg, no, co)


@pytest.mark.parametrize("name,cosmo", [("tiny", False), ("small", True), ("cfg1", False), ("cfg1", True),
                                        ("cfg4s", True)])
def test_snapshot_density(gpu_lib, name, cosmo):
    s = synth.generate(name)
    cfg = s.cfg
    radx, dx = grid.malla(cfg.nx, np.float32(cfg.lado0))
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    g = api.GpuBackend()
    g.upload(s)
    npe = g.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    mesh0 = synth.Mesh(0, np.zeros(1, np.int32), *(np.zeros(0, np.int32) for _ in range(6)),
                       *(np.zeros(0, np.float32) for _ in range(3)), np.zeros(0, np.int32))
    u1, _ = g.density(cfg.nx, np.float32(cfg.lado0), dx, cos["rote"], cos["rete"], npe, mesh0)
    u1, _ = g.renorm_density(cfg.nx, mesh0, np.float32(cfg.fdm), u1, np.zeros((1, abi.NAMRX ** 3), np.float32))
    u1 = np.asarray(u1, np.float32).reshape(cfg.nx, cfg.nx, cfg.nx)
    if cosmo:
        args = (float(cos["contrastec"]), float(cos["rote"]), float(cos["rete"]), float(cos["rodo"]),
                float(cos["re0"]), float(cfg.lado0) / 4, 0.2)
    else:
        args = (200.0, 1.0, 1.0, 1.0, 1.0, 10.0 * float(dx), 0.2)
    ng, cg, no, co = _both(cfg.nx, float(dx), u1, radx, args)
    assert ng > 0
    _same(ng, cg, no, co)


def test_amr_recentering_is_reported_unsupported(gpu_lib):
    nx, lado0 = 32, 32.0
    radx, dx = grid.malla(nx, lado0)
    u = _tophat_field(nx, [((15, 15, 15), 3.0, 400.0)])
    mesh = synth.Mesh(1, np.array([0, 1], np.int32), *(np.array([16], np.int32) for _ in range(3)),
                      *(np.array([12], np.int32) for _ in range(3)),
                      *(np.array([radx[12]], np.float32) for _ in range(3)), np.array([0], np.int32))
    with pytest.raises(api.AsohfError):
        api.GpuBackend().halofind_grid_base(nx, float(dx), u, radx, 200.0, 1.0, 1.0, 1.0, 1.0, 10.0, 0.2,
                                            abi.Catalogue(16), mesh=mesh, u11=np.zeros((1, 32 ** 3), np.float32))
