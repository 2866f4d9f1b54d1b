"""GPU parity of the mesh half of the hot path against the CPU oracle:
species sort, DENSITY, RENORM_DENSITY, INTERPOLATE_DENSITY_TSC, the FFT
Poisson solve and SORT_DM_PARTICLES_X."""
import numpy as np
import pytest

from asohf_b200 import abi, api, grid, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _prep(name, vary_mass=False):
    s = synth.generate(name)
    if vary_mass:  # unequal masses: the general (non-count) deposit paths
        rng = np.random.default_rng(7)
        s.m = (s.m * (1.0 + 0.5 * rng.random(s.m.shape[0]))).astype(np.float32)
    cfg = s.cfg
    radx, dx = grid.malla(cfg.nx, cfg.lado0)
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    return s, cfg, radx, dx, cos


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_species_sort_bit_exact(gpu_lib, name):
    s, cfg, radx, dx, cos = _prep(name)
    g = api.GpuBackend()
    o = O.OracleBackend()
    g.upload(s)
    o.upload(s)
    n_g = g.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    n_o = o.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    assert np.array_equal(n_g, n_o)
    pg, po = g.download(), o.download()
    for f in ["x", "y", "z", "vx", "vy", "vz", "m", "id"]:
        assert np.array_equal(getattr(pg, f), getattr(po, f)), f


@pytest.mark.parametrize("name,vary_mass", [("tiny", False), ("small", False), ("tiny", True),
                                            ("small", True)])
def test_density_matches_fp64_oracle(gpu_lib, name, vary_mass):
    s, cfg, radx, dx, cos = _prep(name, vary_mass)
    g = api.GpuBackend()
    o = O.OracleBackend()
    g.upload(s)
    o.upload(s)
    npe = g.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    o.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    mesh = synth.build_mesh(s, float(dx))
    L = np.float32(cfg.lado0)
    u1g, u11g = g.density(cfg.nx, L, dx, cos["rote"], cos["rete"], npe, mesh)
    u1o, u11o = o.density(cfg.nx, L, dx, cos["rote"], cos["rete"], npe, mesh, fp64=True)
    # base grid: exact sums on both sides -> identical float32
    assert np.array_equal(u1g, u1o)
    # patches: float64 sums in different orders, rounded once
    if mesh.total:
        assert np.allclose(u11g, u11o, rtol=2e-7, atol=0)
    # the reference's own float32 accumulation, for the record
    u1r, _ = o.density(cfg.nx, L, dx, cos["rote"], cos["rete"], npe, mesh, fp64=False)
    assert np.allclose(u1r, u1o, rtol=1e-4)
    # renorm
    fdm = np.float32(cfg.fdm)
    a1, a11 = g.renorm_density(cfg.nx, mesh, fdm, u1g, u11g)
    b1, b11 = o.renorm_density(cfg.nx, mesh, fdm, u1o, u11o)
    assert np.array_equal(a1, b1)


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_tsc_deposit_matches_fp64_oracle(gpu_lib, name):
    s, cfg, radx, dx, cos = _prep(name)
    g = api.GpuBackend()
    o = O.OracleBackend()
    g.upload(s)
    o.upload(s)
    mesh = synth.build_mesh(s, float(dx))
    L = np.float32(cfg.lado0)
    u1g, u11g = g.tsc_deposit(cfg.nx, L, dx, radx, cos["rote"], cos["rete"], mesh)
    u1o, u11o = o.tsc_deposit(cfg.nx, L, dx, radx, cos["rote"], cos["rete"], mesh, fp64=True)
    assert np.allclose(u1g, u1o, rtol=2e-7, atol=1e-30)
    if mesh.total:
        assert np.allclose(u11g, u11o, rtol=2e-7, atol=1e-30)


def _green64(nx, dx):
    """FP64 Green's function of MOMENTO: -(dx/2)^2 / sum sin^2(pi k/N), ~0 at k = 0."""
    k = np.arange(nx)
    s2 = np.sin(np.pi * k / nx) ** 2
    den = s2[:, None, None] + s2[None, :, None] + s2[None, None, :]
    den[0, 0, 0] = 1e30
    return -(float(dx) / 2) ** 2 / den


def _solve64(rho, dx):
    return np.fft.irfftn(np.fft.rfftn(rho.astype(np.float64)) * _green64(rho.shape[0], dx)[..., :rho.shape[0] // 2 + 1],
                         s=rho.shape, axes=(0, 1, 2))


# 16 and 32 take cuFFT 3-D transforms; 64 to 512 cuFFT 2-D transforms of the
# planes around the fused z pass of fftconv.cu
@pytest.mark.parametrize("nx", [16, 32, 64, 128, 256, 512])
def test_poisson_against_fp64_fft(gpu_lib, nx):
    rng = np.random.default_rng(nx)
    rho = rng.standard_normal((nx, nx, nx)).astype(np.float32)
    dx = np.float32(0.37)
    g = api.GpuBackend()
    pot = g.poisson_fft(rho, dx)
    ref = _solve64(rho, dx)
    err = np.abs(pot - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
    if nx <= 256:
        # against the reference's FOURN path (float32 data, float64 twiddles)
        fo = O.poisson_fft(rho, dx)
        err2 = np.abs(pot - fo).max() / np.abs(ref).max()
        assert err2 < 1e-5, err2


@pytest.mark.parametrize("nx", [64, 256])
def test_poisson_batched_copies_are_independent(gpu_lib, nx):
    """A batch of grids of very different magnitudes: every copy is solved on
    its own (no copy's rounding reaches another), each within the FP64 bound."""
    import torch
    rng = np.random.default_rng(7 + nx)
    scales = [1.0, 1e-6, 3e4]
    rho = np.stack([s * rng.standard_normal((nx, nx, nx)) for s in scales]).astype(np.float32)
    dx = np.float32(0.5)
    g = api.GpuBackend()
    r = torch.tensor(rho, device="cuda")
    pot = torch.empty_like(r)
    g.a.poisson_fft(nx, float(dx), r, pot, batch=len(scales))
    torch.cuda.synchronize()
    pot = pot.cpu().numpy()
    for b in range(len(scales)):
        ref = _solve64(rho[b], dx)
        err = np.abs(pot[b] - ref).max() / np.abs(ref).max()
        assert err < 2e-6, (b, err)


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_sort_x_bit_exact(gpu_lib, name):
    s, cfg, radx, dx, cos = _prep(name)
    g = api.GpuBackend()
    o = O.OracleBackend()
    # ties: duplicate some x values so the ARGSORT tie rule is exercised
    s.x[::7] = s.x[3::7][: s.x[::7].shape[0]] if False else s.x[::7]
    x = s.x.copy()
    x[1::5] = x[0::5][: x[1::5].shape[0]]
    x[2::11] = -0.0
    s.x = x
    g.upload(s)
    o.upload(s)
    L = np.float32(cfg.lado0)
    nd_g = g.sort_x(cfg.nx, L)
    nd_o = o.sort_x(cfg.nx, L)
    assert np.array_equal(nd_g, nd_o)
    pg, po = g.download(), o.download()
    for f in ["x", "y", "z", "vx", "vy", "vz", "m", "id"]:
        assert np.array_equal(getattr(pg, f), getattr(po, f)), f
