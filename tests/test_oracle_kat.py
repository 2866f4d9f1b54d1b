"""Known-answer tests of the CPU oracle (no GPU).

The reference ships no tests or fixtures, so these analytic answers are
what pins the oracle: kernel normalisation, mass conservation, cell-centred
clouds, TSC partition of unity, a single Fourier mode through the Poisson
solve, ARGSORT's tie rule, the slab table, and the species sort.
"""
import math

import numpy as np
import pytest

from asohf_b200 import abi, grid, synth
from oracle import oracle as O


@pytest.mark.parametrize("deg", [1, 2])
def test_kernel_normalisation(deg):
    k = O.compute_kernels(6, deg)
    for ir in range(7):
        n = 2 ** ir
        w = k[ir, 512 - n: 512 + n + 1].astype(np.float64)
        s3 = w.sum() ** 3
        # the reference normalises with a REAL*4 sum of (2n+1)^3 products
        # (grids.f:1042-1052): its rounding bounds the residual
        assert abs(s3 - 1.0) < max(2e-6, 6e-8 * (2 * n + 1) ** 3), (ir, s3)
        assert np.allclose(w, w[::-1])


def test_level0_kernel_is_tsc():
    k = O.compute_kernels(0, 2)
    assert list(k[0, 511:514]) == [0.125, 0.75, 0.125]


def test_grid_constants_match_oracle():
    for nx, L in [(32, 14.75), (64, 29.49), (128, 147.5), (256, 368.7)]:
        r1, d1 = grid.malla(nx, L)
        r2, d2 = O.malla(nx, L)
        assert np.array_equal(r1, r2) and d1 == d2
    for h, om, z in [(0.678, 0.31, 0.0), (0.7, 0.3, 1.5)]:
        a, b = grid.cosmology(h, om, z), O.cosmology(h, om, z)
        for key in a:
            assert a[key] == b[key], key


def _mesh0():
    return synth.Mesh(0, np.zeros(1, np.int32), *(np.zeros(0, np.int32) for _ in range(6)),
                      *(np.zeros(0, np.float32) for _ in range(3)), np.zeros(0, np.int32))


def test_density_mass_conservation_and_cell_centre():
    nx, L = 16, 16.0
    radx, dx = grid.malla(nx, L)
    rng = np.random.default_rng(1)
    n = 5000
    x, y, z = (rng.uniform(-L / 2, L / 2, n).astype(np.float32) for _ in range(3))
    m = rng.uniform(0.5, 2.0, n).astype(np.float32)
    b = O.OracleBackend()
    b.p = O.Particles(x, y, z, x, y, z, m, np.arange(n))
    npe = np.zeros(9, np.int32)
    npe[0] = n
    u1, _ = b.density(nx, np.float32(L), dx, np.float32(1.0), np.float32(1.0), npe, _mesh0())
    denbas = np.float32(dx * dx * dx)
    total = float(u1.astype(np.float64).sum() * denbas)
    assert abs(total - float(m.astype(np.float64).sum())) / total < 1e-6
    # one particle at the centre of cell (3,4,5) (1-based)
    c = [radx[3], radx[4], radx[5]]
    xl = np.float32(-L / 2)
    # place it on the cell centre of the DENSITY grid: XL + (I-0.5) DX
    pos = [np.float32(xl + (i - 0.5) * float(dx)) for i in (3, 4, 5)]
    b.p = O.Particles(*[np.array([v], np.float32) for v in pos], *[np.zeros(1, np.float32)] * 3,
                      np.ones(1, np.float32), np.ones(1))
    npe[0] = 1
    u1, _ = b.density(nx, np.float32(L), dx, np.float32(1.0), np.float32(1.0), npe, _mesh0())
    w = [0.125, 0.75, 0.125]
    for kk in range(3):
        for jj in range(3):
            for ii in range(3):
                v = u1[5 - 2 + kk, 4 - 2 + jj, 3 - 2 + ii] * float(denbas)
                assert abs(v - w[ii] * w[jj] * w[kk]) < 1e-6
    del c


def test_tsc_partition_of_unity():
    nx, L = 16, 16.0
    radx, dx = grid.malla(nx, L)
    rng = np.random.default_rng(2)
    b = O.OracleBackend()
    for _ in range(20):
        p = rng.uniform(-L / 2 + 1, L / 2 - 1, 3).astype(np.float32)
        b.p = O.Particles(p[:1], p[1:2], p[2:3], *[np.zeros(1, np.float32)] * 3, np.ones(1, np.float32),
                          np.ones(1))
        u1, _ = b.tsc_deposit(nx, np.float32(L), dx, radx, np.float32(1.0), np.float32(1.0), _mesh0())
        assert abs(u1.astype(np.float64).sum() * float(dx) ** 3 - 1.0) < 1e-5


def test_poisson_single_mode():
    nx = 16
    dx = np.float32(0.5)
    i = np.arange(nx)
    for k in [(1, 0, 0), (2, 3, 1), (0, 0, 5)]:
        rho = (np.cos(2 * np.pi * k[0] * i / nx)[None, None, :]
               * np.cos(2 * np.pi * k[1] * i / nx)[None, :, None]
               * np.cos(2 * np.pi * k[2] * i / nx)[:, None, None]).astype(np.float32)
        pot = O.poisson_fft(rho, dx)
        s2 = sum(math.sin(math.pi * kk / nx) ** 2 for kk in k)
        g = -(float(dx) / 2) ** 2 / s2
        assert np.allclose(pot, g * rho, atol=2e-5 * abs(g)), k


def _merge_argsort_py(a):
    """Transcription of num.f:150-203 (bottom-up merge, right run on ties)."""
    n = len(a)
    indx = list(range(n))
    delta = 1
    while delta < n:
        for iii in range(0, n - delta, 2 * delta):
            i1, i2 = iii, iii + delta
            kkk = min(2 * delta, n - iii)
            tmp = []
            while i1 < iii + delta and i2 < iii + kkk:
                if a[indx[i1]] < a[indx[i2]]:
                    tmp.append(indx[i1]); i1 += 1
                else:
                    tmp.append(indx[i2]); i2 += 1
            tmp += indx[i1:iii + delta] if i1 < iii + delta else indx[i2:iii + kkk]
            indx[iii:iii + kkk] = tmp
        delta *= 2
    return np.array(indx)


@pytest.mark.parametrize("n", [1, 2, 7, 64, 1000, 4097])
def test_argsort_tie_rule(n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, max(2, n // 8), n).astype(np.float32)
    a[rng.random(n) < 0.1] = -0.0
    got = O.argsort(a)
    assert np.array_equal(got, _merge_argsort_py(list(a)))
    # equal keys come out with the larger index first (-0.0 == +0.0)
    keys = np.where(a == 0, 0.0, a)
    assert np.array_equal(got, np.lexsort((-np.arange(n), keys)))


def test_sort_x_slab_table():
    s = synth.generate("tiny")
    L = np.float32(s.cfg.lado0)
    b = O.OracleBackend()
    b.upload(s)
    nd = b.sort_x(s.cfg.nx, L)
    x = b.p.x
    assert np.all(np.diff(x) >= 0)
    xl = np.float32(-L / 2)
    dxl = np.float32(L / np.float32(s.cfg.nx))
    for ix in range(1, s.cfg.nx + 1):
        r = np.float32(xl + np.float32(np.float32(ix) * dxl))
        assert nd[ix] == np.count_nonzero(x <= r)
    assert nd[0] == 0


def test_species_sort_stable_and_formula():
    s = synth.generate("tiny")
    cfg = s.cfg
    radx, dx = grid.malla(cfg.nx, cfg.lado0)
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    b = O.OracleBackend()
    b.upload(s)
    npe = b.species_sort(cfg.nx, dx, cos["rodo"], cos["re0"])
    spec = b.species
    assert npe.sum() == s.x.shape[0]
    # stable: ids (1..N in input order) ascend inside each species block
    ids = b.p.id
    off = 0
    for k in range(abi.N_ESP):
        blk = ids[off: off + npe[k]]
        assert np.all(np.diff(blk) > 0)
        assert np.all(spec[blk - 1] == k)
        off += npe[k]


def test_halo_oracle_finds_generated_haloes():
    from asohf_b200 import driver
    s = synth.generate("tiny")
    r = driver.run(s, O.OracleBackend(), with_subs=False)
    real = r.cat.realclus[: r.cat.nclus] != 0
    assert real.sum() >= 5
    # ID lists: contiguous, disjoint ranges, one entry per bound particle
    ind = r.cat.indcs[: r.cat.nclus][real]
    assert np.all(ind[:, 1] - ind[:, 0] + 1 == r.cat.dmpclus[: r.cat.nclus][real])
    assert len(np.unique(r.pph)) == len(r.pph)


def test_mesh_base_counts_known_answer():
    """CREATE_MESH base counts (grids.f:94-143) on four particles in a 4^3
    grid of side 4: species weights, clamping, border zeroing."""
    from types import SimpleNamespace
    x = np.array([0.5, 0.6, -0.4, 9.0], np.float32)   # cells (3,3,3), (3,3,3), (2,3,3), clamped (4,3,3)
    yz = np.array([0.5, 0.5, 0.5, 0.5], np.float32)
    z0 = np.zeros(4, np.float32)
    o = O.OracleBackend()
    o.upload(SimpleNamespace(x=x, y=yz, z=yz, vx=z0, vy=z0, vz=z0, m=z0 + 1, id=np.arange(4, dtype=np.int32)))
    c = o.mesh_base_counts(4, 1.0, 8, 0, [1, 2]).reshape(4, 4, 4)   # [kz, jy, ix]
    assert c[2, 2, 2] == 1 + 8      # species 0 and species 1
    assert c[2, 2, 1] == 8          # species 1
    assert c[2, 2, 3] == 1          # past the ranges: species 0, clamped to IX = NX
    assert c.sum() == 18
    c = o.mesh_base_counts(4, 1.0, 8, 1, [1, 2]).reshape(4, 4, 4)
    assert c[2, 2, 3] == 0 and c[2, 2, 2] == 9   # IX = NX is a border cell


def test_veinsgrid_reduced_known_answer():
    """VEINSGRID_REDUCED (grids.f:1771-2073): two 8^3 patches of level 1
    overlapping by half in x.  The first marks the half of the second that
    faces it; the second then finds those cells marked and leaves the first
    alone."""
    na = 32
    dx, radx1 = 1.0, -7.5                     # 16 base cells of side 1 from -8
    n = np.array([8, 8], np.int32)
    prx = np.array([-3.5, -1.5], np.float32)  # cell centres of level 0, 4 level-1 cells apart
    pry = prz = np.array([-3.5, -3.5], np.float32)
    cr = np.zeros((2, na, na, na), np.int32)   # [patch, kz, jy, ix]
    cr[:, :8, :8, :8] = 1
    c11 = cr.copy()
    O.OracleBackend().veinsgrid_reduced(1, dx, radx1, n, n, n, prx, pry, prz, 100, cr.reshape(2, -1),
                                        c11.reshape(2, -1))
    assert cr[0, :8, :8, :8].all()              # the first patch is untouched
    assert not cr[1, :8, :8, :4].any()          # the half of the second facing it is zeroed
    assert cr[1, :8, :8, 4:8].all()
    assert np.array_equal(cr, c11)
    with pytest.raises(RuntimeError):            # more neighbours than allowed
        O.OracleBackend().veinsgrid_reduced(1, dx, radx1, n, n, n, prx, pry, prz, 0, cr.reshape(2, -1))


def _tophat_field(nx, spheres):
    """rho/rho_B = 1 with top-hat spheres (centre cell, radius in cells,
    value) whose centre cell is raised by 10 % (a strict peak)."""
    u = np.ones((nx, nx, nx), np.float32)          # [kz, jy, ix]
    k, j, i = np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nx), indexing="ij")
    for (ci, cj, ck), r, v in spheres:
        inside = (i - ci) ** 2 + (j - cj) ** 2 + (k - ck) ** 2 <= r * r
        u[inside] = v
        u[ck, cj, ci] = 1.1 * v
    return u


def test_halofind_grid_base_known_answer():
    """HALOFIND_GRID base level (haloes_grids.f:287-582, no AMR levels): two
    top-hat overdensities give two haloes, the denser first, centred on the
    peak cells; each grows until its mean density falls below CONTRASTEC
    (1 + A (R0/R)^3 = CONTRASTEC gives R = R0 (A/(CONTRASTEC-1))^(1/3))."""
    nx, lado0 = 48, 48.0
    radx, dx = grid.malla(nx, lado0)
    spheres = [((12, 14, 20), 3.0, 400.0), ((34, 30, 26), 4.0, 300.0)]
    u = _tophat_field(nx, spheres)
    cat = abi.Catalogue(64)
    contrastec, rodo, re0 = 200.0, 1.0, 1.0
    n = O.OracleBackend().halofind_grid_base(nx, float(dx), u, radx, contrastec, rodo, re0, rodo, re0,
                                              10.0, 0.2, cat)
    assert n == 2 and cat.nclus == 2
    assert list(cat.realclus[:2]) == [-1, -1] and list(cat.levhal[:2]) == [0, 0]
    for h, ((ci, cj, ck), r0, a) in enumerate(spheres):   # denser sphere first
        assert (cat.clusrx[h], cat.clusry[h], cat.clusrz[h]) == (radx[ci + 1], radx[cj + 1], radx[ck + 1])
        r_pred = r0 * dx * (a / (contrastec - 1.0)) ** (1.0 / 3.0)
        assert 0.85 * r_pred < cat.radio[h] < 1.2 * r_pred
        # mass: the cells inside the final radius, rho_B = 1
        assert cat.masa[h] > a * (4.0 / 3.0) * math.pi * (0.8 * r0) ** 3


def test_halofind_grid_base_recenters_on_a_patch():
    """With an AMR level the new peak moves to the finer level's maximum
    (RECENTER_DENSITY_PEAK, haloes_grids.f:1099-1259): the centre becomes
    that fine cell's RX/RY/RZ and PATCHCLUS the patch."""
    nx, lado0 = 32, 32.0
    radx, dx = grid.malla(nx, lado0)
    u = _tophat_field(nx, [((15, 15, 15), 3.0, 400.0)])     # base peak at RADX(16) = -0.5 on each axis
    na = abi.NAMRX
    # one level-1 patch of 16^3 cells from base cell 12 (PATCHRX = RADX(12) = -4.5)
    mesh = synth.Mesh(1, np.array([0, 1], np.int32), *(np.array([16], np.int32) for _ in range(3)),
                      *(np.array([12], np.int32) for _ in range(3)),
                      *(np.array([radx[12]], np.float32) for _ in range(3)), np.array([0], np.int32))
    k, j, i = np.meshgrid(np.arange(1, na + 1), np.arange(1, na + 1), np.arange(1, na + 1), indexing="ij")
    u11 = (900.0 - 10.0 * ((i - 10) ** 2 + (j - 9) ** 2 + (k - 10) ** 2)).astype(np.float32)[None]
    cat = abi.Catalogue(16)
    n = O.OracleBackend().halofind_grid_base(nx, float(dx), u, radx, 200.0, 1.0, 1.0, 1.0, 1.0, 10.0, 0.2, cat,
                                              mesh=mesh, u11=u11)
    assert n == 1
    # RX(IX) = PATCHRX - DXPA/2 + (IX-1) DXPA with DXPA = 0.5: IX = 10, 9, 10
    assert (cat.clusrx[0], cat.clusry[0], cat.clusrz[0]) == (-0.25, -0.75, -0.25)
    assert cat.patchclus[0] == 1


def test_halofind_grid_amr_known_answer():
    """HALOFIND_GRID on AMR level 1 (haloes_grids.f:586-1097): a top-hat
    overdensity resolved only on a level-1 patch gives one halo of level 1
    on that patch's peak cell, grown over the patch cells (the base cells
    under the patch are masked by CR0AMR) to the top-hat radius."""
    nx, lado0, na = 32, 32.0, abi.NAMRX
    radx, dx = grid.malla(nx, lado0)
    mesh = synth.Mesh(1, np.array([0, 1], np.int32), *(np.array([32], np.int32) for _ in range(3)),
                      *(np.array([9], np.int32) for _ in range(3)),
                      *(np.array([radx[9]], np.float32) for _ in range(3)), np.array([0], np.int32))
    u1 = np.ones((nx, nx, nx), np.float32)
    cr0amr = np.ones((nx, nx, nx), np.int32)
    cr0amr[8:24, 8:24, 8:24] = 0                     # base cells 9..24 lie under the patch
    u11 = _tophat_field(na, [((16, 16, 16), 3.0, 400.0)])[None]   # fine cell 17: RX = 0.25
    ones = np.ones((1, na, na, na), np.int32)
    cat = abi.Catalogue(16)
    n = O.OracleBackend().halofind_grid_amr(1, nx, float(dx), u1, radx, mesh, u11, cr0amr, ones, ones, 200.0,
                                             1.0, 1.0, 1.0, 1.0, 10.0, 0.2, cat)
    assert n == 1 and cat.nclus == 1
    assert (cat.levhal[0], cat.patchclus[0], cat.realclus[0]) == (1, 1, -1)
    assert (cat.clusrx[0], cat.clusry[0], cat.clusrz[0]) == (0.25, 0.25, 0.25)
    r_pred = 3 * 0.5 * (400.0 / 199.0) ** (1.0 / 3.0)
    assert 0.85 * r_pred < cat.radio[0] < 1.2 * r_pred
    # a second call at the same level finds the peak inside the halo: nothing new
    cat2 = abi.Catalogue(16)
    cat2.nclus = 1
    for f in ("clusrx", "clusry", "clusrz", "radio"):
        getattr(cat2, f)[0] = getattr(cat, f)[0]
    cat2.realclus[0] = -1
    assert O.OracleBackend().halofind_grid_amr(1, nx, float(dx), u1, radx, mesh, u11, cr0amr, ones, ones, 200.0,
                                               1.0, 1.0, 1.0, 1.0, 10.0, 0.2, cat2) == 0


def _mesh(nl, npatch, n, px, pr, pare):
    a = lambda v, t=np.int32: np.asarray(v, t)
    return synth.Mesh(nl, a(npatch), a(n[0]), a(n[1]), a(n[2]), a(px[0]), a(px[1]), a(px[2]),
                      a(pr[0], np.float32), a(pr[1], np.float32), a(pr[2], np.float32), a(pare))


def test_compute_cr0amr_known_answer():
    """COMPUTE_CR0AMR (grids.f:2076-2226): base cells under a level-1 patch
    and parent cells under a level-2 child are 0, the rest 1."""
    nx = 16
    radx, dx = grid.malla(nx, 16.0)
    # level 1: 8^3 cells from base cell 3 (covers base 3..6); level 2: 4^3 cells from its cell 2 (covers 2..3)
    r1 = radx[3]
    r2 = r1 - 0.25 + 1 * 0.5          # centre of the parent's cell 2 on level 1 (RX(2) = PATCHRX - DXPA/2 + DXPA)
    m = _mesh(2, [0, 1, 1], ([8, 4], [8, 4], [8, 4]), ([3, 2], [3, 2], [3, 2]), ([r1, r2],) * 3, [0, 1])
    c0, c1 = O.OracleBackend().compute_cr0amr(nx, 16.0, m)
    c0 = c0.reshape(nx, nx, nx)
    assert (c0[2:6, 2:6, 2:6] == 0).all() and c0.sum() == nx ** 3 - 64
    p1 = c1[0].reshape(abi.NAMRX, abi.NAMRX, abi.NAMRX)
    assert (p1[1:3, 1:3, 1:3] == 0).all() and (p1 == 0).sum() == 8
    assert (c1[1] == 1).all()


def test_veinsgrid_known_answer():
    """VEINSGRID (grids.f:2229-2500): two 8^3 patches overlapping by half in
    x; each facing pair keeps one master, the first patch's cell when it is
    not on that patch's faces."""
    na = abi.NAMRX
    m = _mesh(1, [0, 2], ([8, 8], [8, 8], [8, 8]), ([5, 7], [5, 5], [5, 5]),
              ([-3.5, -1.5], [-3.5, -3.5], [-3.5, -3.5]), [0, 0])
    so = np.zeros((2, na ** 3), np.int32)
    O.OracleBackend().veinsgrid(1, 1.0, -7.5, m, so)
    a = so[0].reshape(na, na, na)[:8, :8, :8]
    b = so[1].reshape(na, na, na)[:8, :8, :8]
    assert (a == 0).sum() == 64 + 3 * 28    # A's face cells among the facing ones (ix = 8, or on a y/z face)
    assert (b == 0).sum() == 256 - 148      # the other facing pairs drop B's cell
    assert (a[:, :, :4] == 1).all() and (b[:, :, 4:] == 1).all()


def test_search_substructure_grid_known_answer():
    """SEARCH_SUBSTRUCTURE_GRID (substructure.f:2-697): a top-hat peak on a
    level-1 patch inside a base-level halo becomes one subhalo of that host,
    grown until the Jacobi test R/d > (M/(M + 3 M_host(d)))^(1/3) holds."""
    nx, lado0, na, nb = 32, 32.0, abi.NAMRX, abi.NBINS
    radx, dx = grid.malla(nx, lado0)
    mesh = synth.Mesh(1, np.array([0, 1], np.int32), *(np.array([32], np.int32) for _ in range(3)),
                      *(np.array([9], np.int32) for _ in range(3)),
                      *(np.array([radx[9]], np.float32) for _ in range(3)), np.array([0], np.int32))
    u1 = np.ones((nx, nx, nx), np.float32)
    cr0amr = np.ones((nx, nx, nx), np.int32)
    cr0amr[8:24, 8:24, 8:24] = 0
    u11 = _tophat_field(na, [((24, 16, 16), 3.0, 400.0)])[None]   # fine cell (25, 17, 17): (4.25, 0.25, 0.25)
    ones = np.ones((1, na, na, na), np.int32)
    cat = abi.Catalogue(16)
    cat.nclus = 1                                   # the host, found at level 0
    cat.realclus[0], cat.levhal[0] = -1, 0
    cat.clusrx[0], cat.clusry[0], cat.clusrz[0], cat.radio[0] = -3.75, 0.25, 0.25, 10.0
    r = 0.5 * np.arange(1, nb + 1, dtype=np.float32)
    cat.profiles[0, :nb], cat.profiles[0, nb:] = r, 1000.0 * r   # M_host(r) = 1000 r
    subs_lev = np.array([1, 0], np.int32)
    n = O.OracleBackend().search_substructure_grid(1, nx, float(dx), u1, radx, mesh, u11, cr0amr, ones, ones, 200.0,
                                                    1.0, 1.0, 1.0, 1.0, 1.0, subs_lev, cat)
    assert n == 1 and cat.nclus == 2 and list(subs_lev) == [1, 1]
    assert (cat.realclus[1], cat.levhal[1], cat.patchclus[1]) == (1, 1, 1)
    assert (cat.clusrx[1], cat.clusry[1], cat.clusrz[1]) == (4.25, 0.25, 0.25)
    d, rs, ms = 8.0, float(cat.rsub[1]), float(cat.msub[1])
    assert 1.5 < rs < d
    assert rs / d > (ms / (ms + 3 * 8000.0)) ** (1 / 3)     # the Jacobi test holds at R_SUB
    assert 0 < cat.radio[1] < rs                              # the virial radius comes first
