"""Hot-path driver: the calls PROGRAM ASOHF makes on the particle path
(asohf.f:418-763), in the same order, on a backend (the B200 library, or
any object with the same methods).

Stages outside the hot path are stood in for by asohf_b200.synth: the patch
table (CREATE_MESH) and the halo and subhalo candidates (HALOFIND_GRID,
SEARCH_SUBSTRUCTURE_GRID).  The catalogue cleaning passes CHECK_RUBISH and
ACCIDENTAL_SUBSTRUCTURE are not run.  RE_SORT_HALOES (haloes_particles.f:
2-56), a compaction of the candidate list, is done here on the host.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import abi, grid, synth


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


def re_sort_haloes(cat: abi.Catalogue, nhallev: np.ndarray, ir: int):
    """RE_SORT_HALOES (haloes_particles.f:2-56): drops REALCLUS=0 entries of
    level ir (the last level appended) and renumbers positive REALCLUS."""
    low1 = int(nhallev[:ir].sum()) + 1
    low2 = int(nhallev[: ir + 1].sum())
    j = low1 - 1
    resort = {}
    for i in range(low1, low2 + 1):
        if cat.realclus[i - 1] == 0:
            continue
        j += 1
        resort[i] = j
        for f in ["clusrx", "clusry", "clusrz", "radio", "masa", "levhal", "patchclus", "dmpclus",
                  "clusrxcm", "clusrycm", "clusrzcm"]:
            a = getattr(cat, f)
            a[j - 1] = a[i - 1]
        rc = cat.realclus[i - 1]
        cat.realclus[j - 1] = rc if rc <= 0 else resort.get(int(rc), rc)
    nhallev[ir] = j - (low1 - 1)
    cat.nclus = j


def make_consts(cfg, dx, cos):
    return abi.consts_c(cfg.nx, np.float32(cfg.lado0), dx, cos, np.float32(cfg.fdm),
                        np.float32(cfg.zeta), cfg.min_num_part)


def run(snap: synth.Snapshot, backend, capacity: int | None = None, with_subs: bool = True,
        interp_degree: int = 2) -> RunResult:
    """Runs the hot path on `backend` and returns every stage's output."""
    cfg = snap.cfg
    nx = cfg.nx
    lado0 = np.float32(cfg.lado0)
    radx, dx = grid.malla(nx, lado0)
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    consts = make_consts(cfg, dx, cos)
    T = {}
    from types import SimpleNamespace
    parts = SimpleNamespace(x=snap.x, y=snap.y, z=snap.z, vx=snap.vx, vy=snap.vy, vz=snap.vz,
                            m=snap.m, id=snap.id, n=snap.x.shape[0])
    t0 = time.perf_counter()
    backend.upload(parts)
    T["upload"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    npe = backend.species_sort(nx, dx, cos["rodo"], cos["re0"])
    T["species_sort"] = time.perf_counter() - t0
    mesh = synth.build_mesh(snap, float(dx))
    t0 = time.perf_counter()
    u1, u11 = backend.density(nx, lado0, dx, cos["rote"], cos["rete"], npe, mesh, interp_degree)
    u1, u11 = backend.renorm_density(nx, mesh, np.float32(cfg.fdm), u1, u11)
    T["density"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    nd = backend.sort_x(nx, lado0)
    T["sort_x"] = time.perf_counter() - t0
    cand = synth.build_candidates(snap, mesh, float(dx))
    H = cand.clusrx.shape[0]
    nsub_max = int((snap.halo_host >= 0).sum())
    cap = capacity or (H + nsub_max + 16)
    cat = abi.Catalogue(cap)
    pph = np.zeros(max(snap.x.shape[0], 1), np.int32)
    nhallev = np.zeros(mesh.nl + 1, np.int32)
    base_of_level = np.concatenate([[0], np.cumsum(cand.nhallev)])
    slot_of_truth = {}
    t0 = time.perf_counter()
    for ir in range(mesh.nl + 1):
        lo, hi = int(base_of_level[ir]), int(base_of_level[ir + 1])
        n_new = hi - lo
        if n_new == 0:
            continue
        # HALOFIND_GRID appends the candidates of level ir
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
        truth_slots = list(cand.truth[lo:hi])
        re_sort_haloes(cat, nhallev, ir)
        low1 = int(nhallev[:ir].sum()) + 1
        low2 = int(nhallev[: ir + 1].sum())
        backend.prune_poor_haloes(consts, cat, low1, low2, np.float32(1.0), 1)
        # RE_SORT_HALOES again, keeping track of which truth halo is where
        keep = [t for q, t in enumerate(truth_slots) if cat.realclus[low1 - 1 + q] != 0]
        re_sort_haloes(cat, nhallev, ir)
        low1 = int(nhallev[:ir].sum()) + 1
        low2 = int(nhallev[: ir + 1].sum())
        for q, t in enumerate(keep):
            if t >= 0:
                slot_of_truth[int(t)] = low1 + q
        if nhallev[ir] == 0:
            continue
        backend.halofind_particles(consts, mesh, cat, low1, low2, pph)
        backend.prune_poor_haloes(consts, cat, low1, low2, np.float32(1.0), 0)
    T["halofind"] = time.perf_counter() - t0
    subs_lev = np.zeros(mesh.nl + 1, np.int32)
    subs_lev[0] = cat.nclus
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
    n_ids = int(max([cat.indcs[i, 1] for i in range(cat.nclus) if cat.realclus[i] != 0] + [0]))
    return RunResult(npe, u1, u11, nd, cat, pph[:n_ids].copy(), nhallev, subs_lev,
                     backend.download(), T, mesh)
