"""Seeded synthetic snapshots for the ASOHF particle hot path.

No simulation snapshot or public catalogue is used anywhere.  Particles are
drawn from NFW haloes (mass function dN/dM ~ M^-1.9, concentration
c = 8 (M/1e12)^-0.1, truncated at 2 R200, isotropic Gaussian velocities with
sigma = V200/sqrt(2) plus a bulk velocity) and a uniform background, all from
one numpy PCG64 seed.  Positions and velocities are generated in float64 and
stored as float32, the precision of the reference's generic reader
(readers/particle_general.f:44-64); IDs are 1..N (int32, the reference's
ORIPA).  Units are the reference's code units after reader conversion: cMpc
centred on the box, velocities in units of c, masses in units of
UM = 9.1717e18 Msun (asohf.f:360-361).

Two upstream stages are outside the hot path and are stood in for here:

* ``build_mesh`` places AMR patches around the haloes (the role of
  CREATE_MESH, grids.f:2-707): patches of up to 32^3 cells, aligned to the
  parent grid, PATCHRX = left edge + cell size as in grids.f:300.
* ``build_candidates`` lists halo and subhalo candidates from the generator's
  truth, perturbed, grouped by level (the role of HALOFIND_GRID +
  RE_SORT_HALOES and SEARCH_SUBSTRUCTURE_GRID).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

UM = 9.1717e18          # Msun per code mass unit (asohf.f:361)
UV = 299792.458         # km/s per code velocity unit (asohf.f:360)
GCONS = 4.301e-9        # Mpc km^2 s^-2 Msun^-1


@dataclasses.dataclass
class SnapshotConfig:
    """One synthetic workload.  Sizes follow the benchmark configurations."""
    name: str
    npart_side: int              # N = npart_side**3 particles
    box_mpc_h: float             # box side in Mpc/h
    nx: int                      # base grid cells per side
    nl: int                      # AMR levels
    n_haloes: int
    mlo: float                   # halo mass range, Msun/h
    mhi: float
    frac_haloes: float           # particle fraction in haloes
    sub_host_min: float = 0.0    # hosts above this mass get subhaloes (0: none)
    sub_frac: float = 0.10
    sub_max: int = 8
    sub_conc: float = 15.0
    sub_vkick_kms: float = 200.0
    bulk_kms: float = 300.0
    bg_kms: float = 500.0
    seed: int = 12345
    h: float = 0.678
    omega_m: float = 0.31
    fdm: float = 0.845
    zeta: float = 0.0
    min_num_part: int = 25
    max_patches_per_level: int = 4000

    @property
    def n(self) -> int:
        return self.npart_side ** 3

    @property
    def lado0(self) -> float:
        """Box side in cMpc (the reference's LADO0 after CIO_LENGTH<0)."""
        return self.box_mpc_h / self.h


CONFIGS = {
    # 64^3 particles, 20 Mpc/h, 40 haloes in 1e11-1e13, 64^3 grid, 3 levels
    "cfg1": SnapshotConfig("cfg1", 64, 20.0, 64, 3, 40, 1e11, 1e13, 0.70),
    # 256^3 in 100 Mpc/h, ~5000 haloes in 1e10-1e14 with subhaloes, 6 levels
    "cfg2": SnapshotConfig("cfg2", 256, 100.0, 256, 6, 5000, 1e10, 1e14, 0.65,
                           sub_host_min=1e12),
    # 512^3 in 250 Mpc/h, ~2e5 haloes in 1e10-1e15 (20..1e6 particles)
    "cfg4": SnapshotConfig("cfg4", 512, 250.0, 512, 6, 200000, 1e10, 1e15, 0.70,
                           sub_host_min=1e12),
    # the 512^3 workload at 1/64 of its volume (same density and recipe):
    # the bounded sample the CPU oracle is timed on
    "cfg4s": SnapshotConfig("cfg4s", 128, 62.5, 128, 6, 3125, 1e10, 1e15, 0.70,
                            sub_host_min=1e12),
    # the 512^3 workload at 1/8 of its volume: the second point of the CPU
    # oracle's scaling trend
    "cfg4m": SnapshotConfig("cfg4m", 256, 125.0, 256, 6, 25000, 1e10, 1e15, 0.70,
                            sub_host_min=1e12),
    # small cases for tests
    "tiny": SnapshotConfig("tiny", 32, 10.0, 32, 2, 6, 1e11, 1e12, 0.70,
                           sub_host_min=3e11, seed=7),
    "small": SnapshotConfig("small", 48, 16.0, 48, 3, 25, 1e11, 1e13, 0.70,
                            sub_host_min=1e12, seed=11),
}


@dataclasses.dataclass
class Snapshot:
    cfg: SnapshotConfig
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    m: np.ndarray
    id: np.ndarray
    # truth (float64): haloes then subhaloes
    halo_pos: np.ndarray         # (H, 3) cMpc
    halo_r200: np.ndarray        # (H,) cMpc
    halo_npart: np.ndarray       # (H,)
    halo_host: np.ndarray        # (H,) -1 for a main halo, else index of host


def _nfw_mu(x):
    return np.log1p(x) - x / (1.0 + x)


def _sample_nfw_radius(rng, conc, n_each):
    """Radii (units of R200) from NFW profiles truncated at 2 R200, for a
    batch of haloes: conc[i] with n_each[i] samples each."""
    xs = np.concatenate([[0.0], np.geomspace(1e-5, 2.0 * 40.0, 4000)])
    mu_tab = _nfw_mu(xs)
    cc = np.repeat(conc, n_each)
    u = rng.random(cc.shape[0]) * _nfw_mu(2.0 * cc)
    # invert mu(x) = u on the table (monotone), x in units of r_s
    x = np.interp(u, mu_tab, xs)
    return x / cc


def _random_dirs(rng, n):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v


def generate(cfg: SnapshotConfig | str) -> Snapshot:
    """Generates the particle set of one configuration (deterministic)."""
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    n = cfg.n
    L = cfg.lado0
    h = cfg.h
    # cosmic mean density of DM, Msun / cMpc^3 (rho_crit = 2.775e11 h^2)
    rho_c = 2.775e11 * h * h
    mp_msun = cfg.fdm * cfg.omega_m * rho_c * L ** 3 / n
    # halo masses from dN/dM ~ M^-1.9 on [mlo, mhi] (inverse CDF), Msun/h
    a = -0.9
    u = rng.random(cfg.n_haloes)
    lo, hi = cfg.mlo ** a, cfg.mhi ** a
    mh = (lo + u * (hi - lo)) ** (1.0 / a)
    mh = np.sort(mh)[::-1]
    n_halo_tot = int(round(cfg.frac_haloes * n))
    npart = np.floor(mh / mh.sum() * n_halo_tot).astype(np.int64)
    npart = np.maximum(npart, 1)
    # subhaloes: 10% of qualifying hosts' particles in up to sub_max subs
    sub_host, sub_np = [], []
    if cfg.sub_host_min > 0:
        for i in np.nonzero(mh >= cfg.sub_host_min)[0]:
            ns = int(rng.integers(1, cfg.sub_max + 1))
            take = int(cfg.sub_frac * npart[i])
            if take < 2 * cfg.min_num_part * ns:
                continue
            w = rng.dirichlet(np.ones(ns)) * take
            w = np.maximum(w.astype(np.int64), 1)
            npart[i] -= w.sum()
            sub_host += [i] * ns
            sub_np += list(w)
    sub_host = np.array(sub_host, dtype=np.int64)
    sub_np = np.array(sub_np, dtype=np.int64)
    nbg = n - int(npart.sum()) - int(sub_np.sum())
    assert nbg >= 0
    H = cfg.n_haloes
    # effective halo mass from its particles (truncation at 2 R200)
    conc = 8.0 * (mh / 1e12) ** -0.1
    mtot = npart * mp_msun + np.bincount(sub_host, weights=sub_np * mp_msun, minlength=H)
    m200 = mtot * _nfw_mu(conc) / _nfw_mu(2.0 * conc)
    r200 = (3.0 * m200 / (4.0 * math.pi * 200.0 * rho_c)) ** (1.0 / 3.0)
    v200 = np.sqrt(GCONS * m200 / r200)
    margin = 2.0 * r200
    pos = np.empty((H, 3))
    for d in range(3):
        pos[:, d] = -L / 2 + margin + rng.random(H) * (L - 2 * margin)
    bulk = rng.standard_normal((H, 3)) * cfg.bulk_kms
    # main haloes
    r = _sample_nfw_radius(rng, conc, npart) * np.repeat(r200, npart)
    d = _random_dirs(rng, r.shape[0])
    P = np.repeat(pos, npart, axis=0) + d * r[:, None]
    V = (np.repeat(bulk, npart, axis=0)
         + rng.standard_normal((r.shape[0], 3)) * np.repeat(v200 / math.sqrt(2.0), npart)[:, None])
    parts_p, parts_v = [P], [V]
    # subhaloes
    S = sub_host.shape[0]
    spos = np.zeros((S, 3))
    sr200 = np.zeros(S)
    if S:
        sm200 = sub_np * mp_msun
        sr200 = (3.0 * sm200 / (4.0 * math.pi * 200.0 * rho_c)) ** (1.0 / 3.0)
        sv200 = np.sqrt(GCONS * sm200 / sr200)
        sdist = (0.3 + 0.6 * rng.random(S)) * r200[sub_host]
        spos = pos[sub_host] + _random_dirs(rng, S) * sdist[:, None]
        sbulk = bulk[sub_host] + _random_dirs(rng, S) * cfg.sub_vkick_kms
        sc = np.full(S, cfg.sub_conc)
        rs = _sample_nfw_radius(rng, sc, sub_np) * 0.5 * np.repeat(sr200, sub_np)
        ds = _random_dirs(rng, rs.shape[0])
        parts_p.append(np.repeat(spos, sub_np, axis=0) + ds * rs[:, None])
        parts_v.append(np.repeat(sbulk, sub_np, axis=0)
                       + rng.standard_normal((rs.shape[0], 3))
                       * np.repeat(sv200 / math.sqrt(2.0), sub_np)[:, None])
    # background
    parts_p.append(-L / 2 + rng.random((nbg, 3)) * L)
    parts_v.append(rng.standard_normal((nbg, 3)) * cfg.bg_kms)
    P = np.concatenate(parts_p)
    V = np.concatenate(parts_v) / UV
    # periodic wrap into [-L/2, L/2) and shuffle (file order ~ Lagrangian)
    P = np.mod(P + L / 2, L) - L / 2
    perm = rng.permutation(n)
    P = P[perm].astype(np.float32)
    V = V[perm].astype(np.float32)
    # float32 rounding can land exactly on +L/2: fold back inside
    P[P >= float(np.float32(L / 2))] = float(np.float32(-L / 2))
    m = np.full(n, np.float32(mp_msun / UM), dtype=np.float32)
    ids = np.arange(1, n + 1, dtype=np.int32)
    halo_pos = np.concatenate([pos, spos]) if S else pos
    halo_r200 = np.concatenate([r200, sr200]) if S else r200
    halo_np = np.concatenate([npart, sub_np]) if S else npart
    halo_host = np.concatenate([np.full(H, -1), sub_host]) if S else np.full(H, -1)
    return Snapshot(cfg, np.ascontiguousarray(P[:, 0]), np.ascontiguousarray(P[:, 1]),
                    np.ascontiguousarray(P[:, 2]), np.ascontiguousarray(V[:, 0]),
                    np.ascontiguousarray(V[:, 1]), np.ascontiguousarray(V[:, 2]), m, ids,
                    halo_pos, halo_r200, halo_np, halo_host)


@dataclasses.dataclass
class Mesh:
    """Patch table with the Fortran meaning (1-based levels, NPATCH(0:NL))."""
    nl: int
    npatch: np.ndarray   # int32 (nl+1,)
    patchnx: np.ndarray
    patchny: np.ndarray
    patchnz: np.ndarray
    patchx: np.ndarray
    patchy: np.ndarray
    patchz: np.ndarray
    patchrx: np.ndarray  # float32
    patchry: np.ndarray
    patchrz: np.ndarray
    pare: np.ndarray
    owner: np.ndarray | None = None   # generator halo a stand-in patch was built for

    @property
    def total(self) -> int:
        return int(self.npatch.sum())


def build_mesh(snap: Snapshot, dx: float, nl: int | None = None) -> Mesh:
    """Stand-in for CREATE_MESH: at level ir, one patch (up to 32^3 cells)
    centred on each halo whose particle count and size call for that level,
    largest haloes first, capped per level."""
    cfg = snap.cfg
    nl = cfg.nl if nl is None else nl
    L = cfg.lado0
    H = cfg.n_haloes
    order = np.argsort(-snap.halo_npart[:H], kind="stable")
    rows = []
    npatch = [0]
    for ir in range(1, nl + 1):
        dxpa = dx / 2.0 ** ir
        dxpar = dx / 2.0 ** (ir - 1)
        cnt = 0
        for i in order:
            if snap.halo_npart[i] < 64 * 4 ** (ir - 1):
                break
            rr = snap.halo_r200[i]
            side = int(min(32, max(14, 2 * math.ceil(1.2 * rr / dxpa))))
            side += side % 2
            c = snap.halo_pos[i]
            org = []
            for d in range(3):
                left = c[d] - side * dxpa / 2
                k = math.floor((left + L / 2) / dxpar)  # parent cell index (0-based)
                k = max(0, min(k, int(round(L / dxpar)) - side // 2))
                org.append(k)
            rows.append((ir, side, org, i))
            cnt += 1
            if cnt >= cfg.max_patches_per_level:
                break
        npatch.append(cnt)
    P = len(rows)
    m = Mesh(nl, np.array(npatch, np.int32), *(np.zeros(P, np.int32) for _ in range(6)),
             *(np.zeros(P, np.float32) for _ in range(3)), np.zeros(P, np.int32),
             np.array([r[3] for r in rows], np.int64))
    for q, (ir, side, org, _) in enumerate(rows):
        dxpa = np.float32(dx / 2.0 ** ir)
        dxpar = np.float32(dx / 2.0 ** (ir - 1))
        m.patchnx[q] = m.patchny[q] = m.patchnz[q] = side
        m.patchx[q], m.patchy[q], m.patchz[q] = (k + 1 for k in org)
        left = [np.float32(-L / 2) + np.float32(k) * dxpar for k in org]
        m.patchrx[q], m.patchry[q], m.patchrz[q] = (np.float32(v + dxpa) for v in left)
    return m


@dataclasses.dataclass
class Candidates:
    """Candidate catalogue handed to the particle stage, grouped by level
    (NHALLEV) like RE_SORT_HALOES leaves it."""
    clusrx: np.ndarray
    clusry: np.ndarray
    clusrz: np.ndarray
    radio: np.ndarray
    masa: np.ndarray
    levhal: np.ndarray
    patchclus: np.ndarray
    truth: np.ndarray      # index into the generator's halo list
    nhallev: np.ndarray    # (nl+1,)


def build_candidates(snap: Snapshot, mesh: Mesh, dx: float, seed: int = 99,
                     spurious_frac: float = 0.05) -> Candidates:
    """Stand-in for the grid finder: one candidate per generated main halo
    (centre offset by 0.1 R200 per axis, radius scaled by U(0.7, 1.3)) plus a
    few spurious candidates on the background, grouped by level."""
    cfg = snap.cfg
    rng = np.random.Generator(np.random.PCG64(seed))
    H = cfg.n_haloes
    L = cfg.lado0
    ns = int(spurious_frac * H)
    pos = np.concatenate([snap.halo_pos[:H] + rng.standard_normal((H, 3)) * 0.1 * snap.halo_r200[:H, None],
                          -L / 2 + 0.1 * L + rng.random((ns, 3)) * 0.8 * L])
    rad = np.concatenate([snap.halo_r200[:H] * rng.uniform(0.7, 1.3, H),
                          np.full(ns, 2.0 * dx)])
    truth = np.concatenate([np.arange(H), np.full(ns, -1)])
    lev = np.zeros(H + ns, np.int32)
    pc = np.zeros(H + ns, np.int32)
    # level: the finest level <= the one whose cell is < R/4 that has a patch
    # built around this halo (the grid finder reports a peak on its patch)
    want = np.clip(np.floor(np.log2(np.maximum(dx / np.maximum(rad / 4.0, 1e-9), 1.0))), 0, mesh.nl).astype(int)
    patch_of = {}
    if mesh.owner is not None:
        lev_of_patch = np.repeat(np.arange(mesh.nl + 1), mesh.npatch)
        for q in range(mesh.total):
            patch_of[(int(mesh.owner[q]), int(lev_of_patch[q]))] = q + 1
    for i in range(H):
        for ir in range(int(want[i]), 0, -1):
            q = patch_of.get((i, ir))
            if q is not None:
                lev[i], pc[i] = ir, q
                break
    order = np.argsort(lev, kind="stable")
    mp = float(snap.m[0])
    npart_est = np.concatenate([snap.halo_npart[:H], np.full(ns, 1)])
    return Candidates(pos[order, 0].astype(np.float32), pos[order, 1].astype(np.float32),
                      pos[order, 2].astype(np.float32), rad[order].astype(np.float32),
                      (npart_est[order] * mp * UM).astype(np.float32), lev[order],
                      pc[order], truth[order],
                      np.bincount(lev, minlength=mesh.nl + 1).astype(np.int32))


def build_sub_candidates(snap: Snapshot, host_slot: dict, host_ok, dx: float, nl: int,
                         seed: int = 98):
    """Stand-in for SEARCH_SUBSTRUCTURE_GRID: one candidate per generated
    subhalo whose host survived the halo stage.  host_slot[h] is the 1-based
    catalogue slot of generator halo h (0: none); host_ok(slots) says, for an
    array of slots, which hosts are confirmed haloes.  The centre offsets and
    radius factors are drawn for every generated subhalo (one seeded stream),
    so a candidate's values do not depend on which others are kept.  Returns
    per-candidate arrays, ordered by level (stable), and SUBS_LEV."""
    cfg = snap.cfg
    rng = np.random.Generator(np.random.PCG64(seed))
    H = cfg.n_haloes
    ns = snap.halo_pos.shape[0] - H
    subs_lev = np.zeros(nl + 1, np.int32)
    z = np.zeros(0, np.float32)
    empty = (z, z, z, z, np.zeros(0, np.int32), np.zeros(0, np.int64), subs_lev)
    if ns <= 0:
        return empty
    off = rng.standard_normal((ns, 3))
    fac = rng.uniform(0.8, 1.2, ns)
    idx = np.arange(H, H + ns)
    hosts = np.asarray(snap.halo_host[H:], np.int64)
    hs = np.asarray(host_slot, np.int64)
    inside = (hosts >= 0) & (hosts < hs.shape[0])
    slot = np.zeros(ns, np.int64)
    slot[inside] = hs[hosts[inside]]
    keep = slot > 0
    keep[keep] = np.asarray(host_ok(slot[keep]), bool)
    if not keep.any():
        return empty
    idx, slot, off, fac = idx[keep], slot[keep], off[keep], fac[keep]
    r = np.asarray(snap.halo_r200[idx], np.float64)
    c = np.asarray(snap.halo_pos[idx], np.float64) + off * (0.05 * r)[:, None]
    ratio = np.maximum(dx / np.maximum(r / 2.0, 1e-9), 1.0)
    lev = np.clip(np.floor(np.log2(ratio)).astype(np.int64), 1, nl)
    o = np.argsort(lev, kind="stable")
    lev, c, rad, slot, idx = lev[o], c[o], (r * fac)[o], slot[o], idx[o]
    np.add.at(subs_lev, lev, 1)
    return (c[:, 0].astype(np.float32), c[:, 1].astype(np.float32), c[:, 2].astype(np.float32),
            rad.astype(np.float32), slot.astype(np.int32), idx.astype(np.int64), subs_lev)


def _halo_table(cfg: SnapshotConfig, rng):
    """Per-halo and per-subhalo parameters of the recipe (small arrays)."""
    n = cfg.n
    L = cfg.lado0
    rho_c = 2.775e11 * cfg.h * cfg.h
    mp_msun = cfg.fdm * cfg.omega_m * rho_c * L ** 3 / n
    a = -0.9
    u = rng.random(cfg.n_haloes)
    lo, hi = cfg.mlo ** a, cfg.mhi ** a
    mh = np.sort((lo + u * (hi - lo)) ** (1.0 / a))[::-1]
    npart = np.maximum(np.floor(mh / mh.sum() * int(round(cfg.frac_haloes * n))).astype(np.int64), 1)
    sub_host, sub_np = [], []
    if cfg.sub_host_min > 0:
        for i in np.nonzero(mh >= cfg.sub_host_min)[0]:
            ns = int(rng.integers(1, cfg.sub_max + 1))
            take = int(cfg.sub_frac * npart[i])
            if take < 2 * cfg.min_num_part * ns:
                continue
            w = np.maximum((rng.dirichlet(np.ones(ns)) * take).astype(np.int64), 1)
            npart[i] -= w.sum()
            sub_host += [i] * ns
            sub_np += list(w)
    sub_host = np.array(sub_host, dtype=np.int64)
    sub_np = np.array(sub_np, dtype=np.int64)
    H = cfg.n_haloes
    conc = 8.0 * (mh / 1e12) ** -0.1
    mtot = npart * mp_msun + np.bincount(sub_host, weights=sub_np * mp_msun, minlength=H)
    m200 = mtot * _nfw_mu(conc) / _nfw_mu(2.0 * conc)
    r200 = (3.0 * m200 / (4.0 * math.pi * 200.0 * rho_c)) ** (1.0 / 3.0)
    v200 = np.sqrt(GCONS * m200 / r200)
    margin = 2.0 * r200
    pos = np.empty((H, 3))
    for d in range(3):
        pos[:, d] = -L / 2 + margin + rng.random(H) * (L - 2 * margin)
    bulk = rng.standard_normal((H, 3)) * cfg.bulk_kms
    S = sub_host.shape[0]
    sr200 = np.zeros(S)
    sv200 = np.zeros(S)
    spos = np.zeros((S, 3))
    sbulk = np.zeros((S, 3))
    if S:
        sm200 = sub_np * mp_msun
        sr200 = (3.0 * sm200 / (4.0 * math.pi * 200.0 * rho_c)) ** (1.0 / 3.0)
        sv200 = np.sqrt(GCONS * sm200 / sr200)
        sdist = (0.3 + 0.6 * rng.random(S)) * r200[sub_host]
        spos = pos[sub_host] + _random_dirs(rng, S) * sdist[:, None]
        sbulk = bulk[sub_host] + _random_dirs(rng, S) * cfg.sub_vkick_kms
    return dict(mp=mp_msun, npart=npart, conc=conc, r200=r200, v200=v200, pos=pos, bulk=bulk,
                sub_host=sub_host, sub_np=sub_np, sr200=sr200, sv200=sv200, spos=spos, sbulk=sbulk)


def generate_fast(cfg: SnapshotConfig | str, device: str | None = None, keep_on_device: bool = False):
    """Same recipe as ``generate`` with the per-particle sampling in torch
    (on the GPU when one is present): a 512^3 snapshot in seconds.  The
    random stream differs from ``generate``'s; it is seeded and repeatable
    on a given device type.  With keep_on_device the particle arrays are
    torch tensors on `device`."""
    import torch
    if isinstance(cfg, str):
        cfg = CONFIGS[cfg]
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    rng = np.random.Generator(np.random.PCG64(cfg.seed))
    t = _halo_table(cfg, rng)
    n, L = cfg.n, cfg.lado0
    g = torch.Generator(device=device)
    g.manual_seed(cfg.seed)
    dd = dict(device=device, dtype=torch.float64)
    xs = torch.cat([torch.zeros(1, **dd), torch.logspace(-5, math.log10(80.0), 4000, **dd)])
    mu_tab = torch.log1p(xs) - xs / (1.0 + xs)

    def nfw_r(conc, counts, scale):
        c = torch.repeat_interleave(torch.as_tensor(conc, **dd), torch.as_tensor(counts, device=device))
        mu_max = torch.log1p(2.0 * c) - 2.0 * c / (1.0 + 2.0 * c)
        u = torch.rand(c.shape[0], generator=g, **dd) * mu_max
        k = torch.clamp(torch.searchsorted(mu_tab, u), 1, xs.shape[0] - 1)
        x0, x1, m0, m1 = xs[k - 1], xs[k], mu_tab[k - 1], mu_tab[k]
        x = x0 + (u - m0) * (x1 - x0) / torch.clamp(m1 - m0, min=1e-300)
        s = torch.repeat_interleave(torch.as_tensor(scale, **dd), torch.as_tensor(counts, device=device))
        return x / c * s

    def dirs(m):
        v = torch.randn(m, 3, generator=g, **dd)
        return v / torch.linalg.norm(v, dim=1, keepdim=True)

    def rep(a, counts):
        return torch.repeat_interleave(torch.as_tensor(a, **dd), torch.as_tensor(counts, device=device), dim=0)

    r = nfw_r(t["conc"], t["npart"], t["r200"])
    P = [rep(t["pos"], t["npart"]) + dirs(r.shape[0]) * r[:, None]]
    V = [rep(t["bulk"], t["npart"]) + torch.randn(r.shape[0], 3, generator=g, **dd)
         * rep(t["v200"] / math.sqrt(2.0), t["npart"])[:, None]]
    del r
    S = t["sub_host"].shape[0]
    if S:
        rs = nfw_r(np.full(S, cfg.sub_conc), t["sub_np"], 0.5 * t["sr200"])
        P.append(rep(t["spos"], t["sub_np"]) + dirs(rs.shape[0]) * rs[:, None])
        V.append(rep(t["sbulk"], t["sub_np"]) + torch.randn(rs.shape[0], 3, generator=g, **dd)
                 * rep(t["sv200"] / math.sqrt(2.0), t["sub_np"])[:, None])
        del rs
    nbg = n - int(t["npart"].sum()) - int(t["sub_np"].sum())
    P.append(-L / 2 + torch.rand(nbg, 3, generator=g, **dd) * L)
    V.append(torch.randn(nbg, 3, generator=g, **dd) * cfg.bg_kms)
    P = torch.remainder(torch.cat(P) + L / 2, L) - L / 2
    V = torch.cat(V) / UV
    perm = torch.randperm(n, generator=g, device=device)
    P = P[perm].to(torch.float32)
    V = V[perm].to(torch.float32)
    del perm
    P[P >= float(np.float32(L / 2))] = float(np.float32(-L / 2))
    m = torch.full((n,), float(np.float32(t["mp"] / UM)), dtype=torch.float32, device=device)
    ids = torch.arange(1, n + 1, dtype=torch.int32, device=device)
    cols = [P[:, 0].contiguous(), P[:, 1].contiguous(), P[:, 2].contiguous(), V[:, 0].contiguous(),
            V[:, 1].contiguous(), V[:, 2].contiguous(), m, ids]
    del P, V
    if not keep_on_device:
        cols = [c.cpu().numpy() for c in cols]
    H = cfg.n_haloes
    halo_pos = np.concatenate([t["pos"], t["spos"]]) if S else t["pos"]
    halo_r200 = np.concatenate([t["r200"], t["sr200"]]) if S else t["r200"]
    halo_np = np.concatenate([t["npart"], t["sub_np"]]) if S else t["npart"]
    halo_host = np.concatenate([np.full(H, -1), t["sub_host"]]) if S else np.full(H, -1)
    return Snapshot(cfg, *cols, halo_pos, halo_r200, halo_np, halo_host)
