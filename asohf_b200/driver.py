"""Hot-path driver: the calls PROGRAM ASOHF makes on the particle path
(asohf.f:418-763), in the same order, on a backend (the B200 library, or
any object with the same methods).

Stages outside the hot path are stood in for by asohf_b200.synth and
prepared before the hot path runs (``prepare``): the patch table
(CREATE_MESH) and the halo candidates (HALOFIND_GRID).  Subhalo candidates
(SEARCH_SUBSTRUCTURE_GRID) are listed during the run, once the host haloes
are known.  The catalogue cleaning passes CHECK_RUBISH and
ACCIDENTAL_SUBSTRUCTURE run on the backend after each level's refinement,
as asohf.f:669-675 calls them.  RE_SORT_HALOES (haloes_particles.f:2-56),
a compaction of the candidate list, is done here on the host.
"""
from __future__ import annotations

import dataclasses
import time
from types import SimpleNamespace

import numpy as np

from . import abi, grid, synth


@dataclasses.dataclass
class Plan:
    snap: synth.Snapshot
    radx: np.ndarray
    dx: np.float32
    cos: dict
    consts: abi.ConstsC
    mesh: synth.Mesh
    cand: synth.Candidates
    capacity: int


@dataclasses.dataclass
class RunResult:
    npart_esp: np.ndarray
    u1: np.ndarray
    u11: np.ndarray
    ndmpart_x: np.ndarray
    cat: abi.Catalogue
    pph: np.ndarray
    nhallev: np.ndarray
    subs_lev: np.ndarray
    particles: object
    stage_s: dict
    mesh: object


CAT_MOVE = ["clusrx", "clusry", "clusrz", "radio", "masa", "levhal", "patchclus", "dmpclus",
            "clusrxcm", "clusrycm", "clusrzcm"]


def re_sort_haloes(cat: abi.Catalogue, nhallev: np.ndarray, ir: int):
    """RE_SORT_HALOES (haloes_particles.f:2-56): drops REALCLUS=0 entries of
    level ir (the last level appended), keeping order, and renumbers
    positive REALCLUS through the old->new map."""
    low1 = int(nhallev[:ir].sum()) + 1
    low2 = int(nhallev[: ir + 1].sum())
    sl = slice(low1 - 1, low2)
    rc = cat.realclus[sl].copy()
    keep = rc != 0
    idx = np.flatnonzero(keep)
    k = int(idx.shape[0])
    if k == low2 - low1 + 1:  # nothing dropped: order and numbering stay
        nhallev[ir] = k
        cat.nclus = low1 - 1 + k
        return keep
    resort = np.zeros(low2 - low1 + 1, np.int64)
    resort[idx] = np.arange(low1, low1 + k)
    for f in CAT_MOVE:
        a = getattr(cat, f)
        a[low1 - 1: low1 - 1 + k] = np.take(a[sl], idx)
    new = rc[idx]
    pos = new > 0
    inside = pos & (new >= low1) & (new <= low2)
    new[inside] = resort[new[inside] - low1]
    cat.realclus[low1 - 1: low1 - 1 + k] = new
    nhallev[ir] = k
    cat.nclus = low1 - 1 + k
    return keep


def make_consts(cfg, dx, cos):
    return abi.consts_c(cfg.nx, np.float32(cfg.lado0), dx, cos, np.float32(cfg.fdm),
                        np.float32(cfg.zeta), cfg.min_num_part)


def prepare(snap: synth.Snapshot, capacity: int | None = None) -> Plan:
    cfg = snap.cfg
    radx, dx = grid.malla(cfg.nx, cfg.lado0)
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    mesh = synth.build_mesh(snap, float(dx))
    cand = synth.build_candidates(snap, mesh, float(dx))
    nsub = int((snap.halo_host >= 0).sum())
    cap = capacity or (cand.clusrx.shape[0] + nsub + 16)
    return Plan(snap, radx, dx, cos, make_consts(cfg, dx, cos), mesh, cand, cap)


def execute(plan: Plan, backend, with_subs: bool = True, interp_degree: int = 2,
            particles=None, download: bool = True) -> RunResult:
    """Runs the hot path on `backend`; returns every stage's output."""
    snap, cfg = plan.snap, plan.snap.cfg
    nx, lado0, dx, cos, consts, mesh, cand = (cfg.nx, np.float32(cfg.lado0), plan.dx, plan.cos,
                                              plan.consts, plan.mesh, plan.cand)
    T = {}
    parts = particles or SimpleNamespace(x=snap.x, y=snap.y, z=snap.z, vx=snap.vx, vy=snap.vy,
                                         vz=snap.vz, m=snap.m, id=snap.id, n=snap.x.shape[0])
    t0 = time.perf_counter()
    backend.upload(parts)
    T["upload"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    npe = backend.species_sort(nx, dx, cos["rodo"], cos["re0"])
    T["species_sort"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    if hasattr(backend, "density_renorm"):  # one transfer of the grids
        u1, u11 = backend.density_renorm(nx, lado0, dx, cos["rote"], cos["rete"], npe, mesh, interp_degree,
                                         np.float32(cfg.fdm))
    else:
        u1, u11 = backend.density(nx, lado0, dx, cos["rote"], cos["rete"], npe, mesh, interp_degree)
        u1, u11 = backend.renorm_density(nx, mesh, np.float32(cfg.fdm), u1, u11)
    T["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    nd = backend.sort_x(nx, lado0)
    T["sort_x"] = time.perf_counter() - t0
    if hasattr(backend, "catalogue"):  # backend-owned page-locked catalogues, reused
        cat = backend.catalogue(plan.capacity)
    else:
        cat = abi.Catalogue(plan.capacity, pinned=getattr(backend, "pinned_host", False))
    n_id_cap = max(snap.x.shape[0], 1)
    pph = np.zeros(n_id_cap, np.int32)
    nhallev = np.zeros(mesh.nl + 1, np.int32)
    base_of_level = np.concatenate([[0], np.cumsum(cand.nhallev)])
    slot_of_truth = np.zeros(max(int(snap.halo_pos.shape[0]), 1), np.int64)  # generator halo -> slot
    t0 = time.perf_counter()
    for ir in range(mesh.nl + 1):
        lo, hi = int(base_of_level[ir]), int(base_of_level[ir + 1])
        n_new = hi - lo
        if n_new == 0:
            continue
        s0 = cat.nclus
        sl = slice(s0, s0 + n_new)
        cat.clusrx[sl] = cand.clusrx[lo:hi]
        cat.clusry[sl] = cand.clusry[lo:hi]
        cat.clusrz[sl] = cand.clusrz[lo:hi]
        cat.radio[sl] = cand.radio[lo:hi]
        cat.masa[sl] = cand.masa[lo:hi]
        cat.levhal[sl] = cand.levhal[lo:hi]
        cat.patchclus[sl] = cand.patchclus[lo:hi]
        cat.realclus[sl] = -1
        cat.nclus = s0 + n_new
        nhallev[ir] = n_new
        truth = cand.truth[lo:hi]
        resort = getattr(backend, "re_sort_haloes", re_sort_haloes)
        truth = truth[resort(cat, nhallev, ir)]
        low1 = int(nhallev[:ir].sum()) + 1
        low2 = int(nhallev[: ir + 1].sum())
        backend.prune_poor_haloes(consts, cat, low1, low2, np.float32(1.0), 1)
        truth = truth[resort(cat, nhallev, ir)]
        low1 = int(nhallev[:ir].sum()) + 1
        low2 = int(nhallev[: ir + 1].sum())
        known = truth >= 0
        slot_of_truth[truth[known]] = low1 + np.nonzero(known)[0]
        if nhallev[ir] == 0:
            continue
        backend.halofind_particles(consts, mesh, cat, low1, low2, pph)
        backend.prune_poor_haloes(consts, cat, low1, low2, np.float32(1.0), 0)
        # catalogue cleaning (asohf.f:672-675)
        backend.check_rubish(cat, low1, low2)
        backend.accidental_substructure(cat)
    T["halofind"] = time.perf_counter() - t0
    subs_lev = np.zeros(mesh.nl + 1, np.int32)
    subs_lev[0] = cat.nclus
    nsub_max = int((snap.halo_host >= 0).sum())
    if with_subs and nsub_max > 0 and mesh.nl >= 1:
        t0 = time.perf_counter()
        sx, sy, sz, srad, shost, struth, slev = synth.build_sub_candidates(
            snap, slot_of_truth, lambda s: cat.realclus[s - 1] == -1, float(dx), mesh.nl)
        base = np.concatenate([[0], np.cumsum(slev[1:])])
        for ir in range(1, mesh.nl + 1):
            lo, hi = int(base[ir - 1]), int(base[ir])
            n_new = hi - lo
            subs_lev[ir] = n_new
            if n_new == 0:
                continue
            s0 = cat.nclus
            sl = slice(s0, s0 + n_new)
            cat.clusrx[sl] = sx[lo:hi]
            cat.clusry[sl] = sy[lo:hi]
            cat.clusrz[sl] = sz[lo:hi]
            cat.rsub[sl] = srad[lo:hi]
            cat.realclus[sl] = shost[lo:hi]
            cat.levhal[sl] = ir
            cat.patchclus[sl] = 0
            cat.nclus = s0 + n_new
            backend.substructure_particles(consts, mesh, cat, ir, subs_lev, pph)
        T["substructure"] = time.perf_counter() - t0
    live = cat.realclus[: cat.nclus] != 0
    n_ids = int(cat.indcs[: cat.nclus][live][:, 1].max()) if live.any() else 0
    ids = backend.final_ids(pph, n_ids)
    if hasattr(backend, "sync_outputs"):  # host grids copied while the halo finder ran
        backend.sync_outputs()
    return RunResult(npe, u1, u11, nd, cat, ids, nhallev, subs_lev,
                     backend.download() if download else None, T, mesh)


def run(snap: synth.Snapshot, backend, capacity: int | None = None, with_subs: bool = True,
        interp_degree: int = 2) -> RunResult:
    """prepare + execute."""
    return execute(prepare(snap, capacity), backend, with_subs=with_subs, interp_degree=interp_degree)
