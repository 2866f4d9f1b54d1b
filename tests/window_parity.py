"""Catalogue parity on a window of haloes, for workloads where running the
oracle on every halo would take too long (the 512^3 benchmark snapshot).

Each halo of HALOFIND_PARTICLES (haloes_particles.f:740-1353) and each
subhalo of SUBSTRUCTURE_PARTICLES (substructure.f:876-1660) is refined from
its own catalogue row, the x-sorted particle store and, for a subhalo, its
host's row; rows do not depend on one another.  So a ``Recorder`` wraps the
device backend and keeps, for every call, the catalogue as the call received
it and as the call left it, plus the bound-ID lists the call wrote.
``run_oracle_rows`` then reruns the oracle on the same x-sorted store for a
chosen set of rows of each call (the others masked out with REALCLUS = 0)
and ``compare_rows`` compares those rows field by field and their ID lists
element by element, with the oracle's decision-margin counts (particle
tests within a relative 1e-6 of their threshold) reported beside the
result.  Float tolerances are those of catalogue_compare: 1e-5 relative,
and for sums of signed terms 1e-5 of the field's largest magnitude.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from asohf_b200 import abi
from oracle import oracle as O
from tests.catalogue_compare import FLOAT_FIELDS

INT_FIELDS_ROW = ["realclus", "dmpclus", "iplip"]
SIGNED_SUM_FIELDS = ("mean_vr", "angularm", "vx", "vy", "vz", "inertia_tensor")


@dataclasses.dataclass
class Call:
    kind: str          # "halo" or "sub"
    low1: int          # 1-based first row of the call
    low2: int          # 1-based last row
    ir: int            # level (subhalo calls)
    subs_lev: np.ndarray
    pre: abi.Catalogue
    post: abi.Catalogue
    ids: np.ndarray    # ID stream slice [id_lo, id_lo + len) written by the call
    id_lo: int


class Recorder:
    """Forwards every method to `backend`; records the refinement calls."""

    def __init__(self, backend):
        self._b = backend
        self.calls: list[Call] = []

    def __getattr__(self, name):
        return getattr(self._b, name)

    def _stream(self, post, low1, low2, pph):
        live = post.realclus[low1 - 1:low2] != 0
        if not live.any():
            return np.zeros(0, np.int32), 0
        ind = post.indcs[low1 - 1:low2][live]
        lo, hi = int(ind[:, 0].min()), int(ind[:, 1].max())
        a = getattr(self._b, "a", None)
        if a is None:  # a host backend (the oracle) writes the driver's array
            return np.asarray(pph[lo - 1:hi]).copy(), lo
        try:
            import torch
            if torch.cuda.is_available():
                buf = torch.empty(max(hi, 1), dtype=torch.int32, device=f"cuda:{a.device}")
                s = a.particles_per_halo(buf)
                return s[lo - 1:hi].cpu().numpy().copy(), lo
        except ImportError:
            pass
        s = a.particles_per_halo()
        return np.asarray(s[lo - 1:hi]).copy(), lo

    def halofind_particles(self, consts, mesh, cat, low1, low2, pph):
        pre = cat.copy()
        self._b.halofind_particles(consts, mesh, cat, low1, low2, pph)
        ids, lo = self._stream(cat, low1, low2, pph)
        self.calls.append(Call("halo", low1, low2, 0, np.zeros(0, np.int32), pre, cat.copy(), ids, lo))

    def substructure_particles(self, consts, mesh, cat, ir, subs_lev, pph):
        sl = np.asarray(subs_lev, np.int32).copy()
        low1 = int(sl[:ir].sum()) + 1
        low2 = int(sl[:ir + 1].sum())
        pre = cat.copy()
        self._b.substructure_particles(consts, mesh, cat, ir, subs_lev, pph)
        ids, lo = self._stream(cat, low1, low2, pph)
        self.calls.append(Call("sub", low1, low2, ir, sl, pre, cat.copy(), ids, lo))


def choose_rows(call: Call, rng, n_random=200, n_largest=20, tier_min=32768):
    """0-based rows of the call to check: the n_largest by the device's bound
    count, every row at or above tier_min members (the thread-block-cluster
    tier), and n_random others drawn with `rng`."""
    rows = np.arange(call.low1 - 1, call.low2)
    rows = rows[call.pre.realclus[rows] != 0]
    if rows.size == 0:
        return rows
    size = call.post.dmpclus[rows].astype(np.int64)
    pick = set(rows[np.argsort(-size, kind="stable")[:n_largest]].tolist())
    pick |= set(rows[size >= tier_min].tolist())
    rest = np.array(sorted(set(rows.tolist()) - pick), np.int64)
    if rest.size:
        pick |= set(rng.choice(rest, size=min(n_random, rest.size), replace=False).tolist())
    return np.array(sorted(pick), np.int64)


class OracleStore:
    """The oracle's view (orc_store) of an x-sorted particle store."""

    def __init__(self, x, y, z, vx, vy, vz, m, ids, ndmpart_x):
        self.arrays = [np.ascontiguousarray(a, np.float32) for a in (x, y, z, vx, vy, vz, m)]
        self.ids = np.ascontiguousarray(ids, np.int32)
        self.nd = np.ascontiguousarray(ndmpart_x, np.int32)
        s = O.StoreC()
        s.n = self.ids.shape[0]
        s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m = (O.P(a) for a in self.arrays)
        s.id = O.P(self.ids, O._ip)
        s.ndmpart_x = O.P(self.nd, O._ip)
        s.norma = float(self.arrays[6].max())
        self.c = s


def run_oracle_rows(call: Call, rows, store: OracleStore, consts, mesh, nthreads=0):
    """Reruns the oracle for `rows` of `call`; returns (catalogue, ID
    stream, margin counts)."""
    import ctypes as C
    cat = call.pre.copy()
    keep = np.zeros(cat.capacity, bool)
    keep[rows] = True
    rng_rows = np.arange(call.low1 - 1, call.low2)
    cat.realclus[rng_rows[~keep[rng_rows]]] = 0
    cat.indcs[:call.low1 - 1] = 0      # the oracle's ID stream starts at this call
    cap = int(call.post.dmpclus[rows].astype(np.int64).sum() * 2 + 1_000_000)
    pph = np.zeros(cap, np.int32)
    n = C.c_int64()
    mh = abi.MeshHolder(mesh)
    cc = cat.as_c()
    nth = C.c_int(nthreads or (__import__("os").cpu_count() or 1))
    margins = O.MarginCounts(cat.capacity)
    with margins:
        if call.kind == "halo":
            rc = O.lib().orc_halofind_particles(C.byref(store.c), C.byref(consts), C.byref(mh.c), C.byref(cc),
                                                C.c_int(call.low1), C.c_int(call.low2), O.P(pph, O._ip),
                                                C.c_int64(cap), C.byref(n), nth)
        else:
            rc = O.lib().orc_substructure_particles(C.byref(store.c), C.byref(consts), C.byref(mh.c),
                                                    C.byref(cc), C.c_int(call.ir), O.P(call.subs_lev, O._ip),
                                                    O.P(pph, O._ip), C.c_int64(cap), C.byref(n), nth)
    if rc:
        raise RuntimeError(f"oracle {call.kind} level call failed: {abi.ERRORS.get(rc, rc)}")
    return cat, pph[:n.value], margins


def compare_rows(call: Call, rows, ocat, opph, margins, rtol=1e-5):
    """Field-by-field and ID-by-ID comparison of `rows`; returns a report.
    A row that differs is acceptable only if the oracle counted a decision
    within 1e-6 of its threshold in it (listed under 'explained')."""
    g = call.post
    bad_rows = {}
    for f in INT_FIELDS_ROW:
        d = rows[getattr(g, f)[rows] != getattr(ocat, f)[rows]]
        for r in d:
            bad_rows.setdefault(int(r), []).append(f)
    for f in FLOAT_FIELDS:
        a = getattr(g, f)[rows].astype(np.float64)
        b = getattr(ocat, f)[rows].astype(np.float64)
        if f in SIGNED_SUM_FIELDS:
            tol = rtol * max(float(np.abs(b).max(initial=0.0)), 1e-30)
        else:
            tol = rtol * np.maximum(np.abs(b), 1e-30) + 1e-30
        over = np.abs(a - b) > tol
        if over.ndim > 1:
            over = over.reshape(over.shape[0], -1).any(axis=1)
        for r in rows[over]:
            bad_rows.setdefault(int(r), []).append(f)
    n_ids = 0
    for r in rows:
        if g.realclus[r] == 0 or ocat.realclus[r] == 0:
            continue
        gs, ge = int(g.indcs[r, 0]), int(g.indcs[r, 1])
        os_, oe = int(ocat.indcs[r, 0]), int(ocat.indcs[r, 1])
        gi = call.ids[gs - call.id_lo: ge - call.id_lo + 1]
        oi = opph[os_ - 1: oe]
        n_ids += oi.shape[0]
        if not np.array_equal(gi, oi):
            bad_rows.setdefault(int(r), []).append("ids")
    near = margins.rows[rows].sum(axis=1)
    explained = {r: v for r, v in bad_rows.items() if margins.rows[r].sum() > 0}
    unexplained = {r: v for r, v in bad_rows.items() if r not in explained}
    return {
        "kind": call.kind, "low1": call.low1, "low2": call.low2, "rows": int(rows.size),
        "bound_ids": n_ids, "margins": margins.totals(rows), "rows_with_margin": int((near > 0).sum()),
        "explained": explained, "unexplained": unexplained,
    }
