"""Python binding of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE ONLY.

The oracle is a C restatement of the reference Fortran routines of the
particle hot path (oracle_grid.c, oracle_halo.c).  Only tests/, the smoke
check and bench.py's CPU-baseline leg use it, as the checker.  Parity status:
unpinned by the reference (no Fortran compiler here, no reference tests or
fixtures); pinned by analytic known-answer tests and committed golden vectors.

``OracleBackend`` exposes the same methods as the GPU backend
(asohf_b200.api.GpuBackend) so one driver (asohf_b200.driver) runs either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from asohf_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class CosmoC(C.Structure):
    _fields_ = [(f, C.c_float) for f in
                ["pi", "ache", "rodo", "re0", "cgr", "rote", "rete", "uv", "um",
                 "contrastec", "omegaz"]]


class StoreC(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", _fp), ("y", _fp), ("z", _fp), ("vx", _fp),
                ("vy", _fp), ("vz", _fp), ("m", _fp), ("id", _ip), ("ndmpart_x", _ip),
                ("norma", C.c_float)]


def build():
    """Compiles liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        srcs = [os.path.join(_HERE, f) for f in ("oracle_grid.c", "oracle_halo.c", "oracle.h")]
        if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in srcs):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_species_sort.restype = C.c_int
        _LIB.orc_halofind_particles.restype = C.c_int
        _LIB.orc_substructure_particles.restype = C.c_int
    return _LIB


def P(a, t=_fp):
    return a.ctypes.data_as(t)


def malla(nx, lado0):
    radx = np.zeros(nx + 2, np.float32)
    dx = C.c_float()
    lib().orc_malla(C.c_int(nx), C.c_float(lado0), P(radx), C.byref(dx))
    return radx, np.float32(dx.value)


def cosmology(h, omega0, zeta):
    c = CosmoC()
    lib().orc_cosmology(C.c_float(h), C.c_float(omega0), C.c_float(zeta), C.byref(c))
    return {f: np.float32(getattr(c, f)) for f, _ in CosmoC._fields_}


def compute_kernels(nl, interp_degree=2):
    W = 2 * 512 + 1
    k = np.zeros((abi.NLEVELS + 1, W), np.float32)
    lib().orc_compute_kernels(C.c_int(nl), C.c_int(interp_degree), P(k))
    return k


def argsort(a):
    a = np.ascontiguousarray(a, np.float32)
    idx = np.zeros(a.shape[0], np.int64)
    lib().orc_argsort(C.c_int64(a.shape[0]), P(a), P(idx, _lp))
    return idx - 1


def momento(nx, dx):
    k = np.zeros(nx ** 3, np.float32)
    lib().orc_momento(C.c_int(nx), C.c_float(dx), P(k))
    return k.reshape(nx, nx, nx)  # [k][j][i]


def poisson_fft(u1, dx):
    nx = u1.shape[0]
    u1 = np.ascontiguousarray(u1, np.float32)
    pot = np.zeros_like(u1)
    lib().orc_poisson_fft(C.c_int(nx), C.c_float(dx), P(u1), P(pot))
    return pot


class Particles:
    """Host SoA particle arrays (owned copies)."""

    def __init__(self, x, y, z, vx, vy, vz, m, id):
        f = lambda a: np.ascontiguousarray(a, np.float32).copy()
        self.x, self.y, self.z = f(x), f(y), f(z)
        self.vx, self.vy, self.vz = f(vx), f(vy), f(vz)
        self.m = f(m)
        self.id = np.ascontiguousarray(id, np.int32).copy()

    @property
    def n(self):
        return self.x.shape[0]

    def ptrs(self):
        return (P(self.x), P(self.y), P(self.z), P(self.vx), P(self.vy), P(self.vz), P(self.m),
                P(self.id, _ip))

    @classmethod
    def from_snapshot(cls, s):
        return cls(s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m, s.id)


class MarginCounts:
    """Decision-margin counts of the oracle's halo and subhalo refinement
    (orc_set_margin_counts): per catalogue row, the particle tests within a
    relative 1e-6 of their threshold -- [0] growth-sphere membership,
    [1] overdensity (virial index, SO walk, subhalo Jacobi estimate),
    [2] escape energy (UNBINDING8), [3] velocity dispersion
    (UNBINDING_SIGMA).  Use as a context manager around the oracle calls."""

    KINDS = ("membership", "overdensity", "escape_energy", "dispersion")

    def __init__(self, capacity: int):
        self.rows = np.zeros((int(capacity), 4), np.int32)

    def __enter__(self):
        lib().orc_set_margin_counts(P(self.rows, _ip), C.c_int64(self.rows.shape[0]))
        return self

    def __exit__(self, *exc):
        lib().orc_set_margin_counts(None, C.c_int64(0))
        return False

    def totals(self, rows=None) -> dict:
        r = self.rows if rows is None else self.rows[rows]
        t = r.sum(axis=0)
        return {k: int(v) for k, v in zip(self.KINDS, t)}


class OracleBackend:
    """Runs each hot-path routine on the CPU oracle.  Methods mirror the
    reference subroutines; arrays are numpy, Fortran layouts."""

    name = "oracle"

    def __init__(self, nthreads: int = 0):
        self.nthreads = nthreads or (os.cpu_count() or 1)
        self.p = None
        self.ndmpart_x = None

    # particle store
    def upload(self, parts):
        self.p = Particles(parts.x, parts.y, parts.z, parts.vx, parts.vy, parts.vz, parts.m, parts.id)

    def download(self) -> Particles:
        return self.p

    def species_sort(self, nx, dx, rodo, re0):
        p = self.p
        npe = np.zeros(abi.N_ESP, np.int32)
        spec = np.zeros(p.n, np.int32)
        rc = lib().orc_species_sort(C.c_int64(p.n), *p.ptrs(), C.c_int(nx), C.c_float(dx),
                                    C.c_float(rodo), C.c_float(re0), P(npe, _ip), P(spec, _ip))
        if rc:
            raise RuntimeError(abi.ERRORS[rc])
        self.species = spec
        return npe

    def density(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree=2, fp64=True):
        p = self.p
        mh = abi.MeshHolder(mesh)
        u1 = np.zeros(nx ** 3, np.float32)
        u11 = np.zeros((max(mesh.total, 1), abi.NAMRX ** 3), np.float32)
        lib().orc_density(C.c_int(nx), C.c_float(lado0), C.c_float(dx), C.c_float(rote),
                          C.c_float(rete), P(p.x), P(p.y), P(p.z), P(p.m),
                          P(np.ascontiguousarray(npart_esp, np.int32), _ip), C.byref(mh.c),
                          C.c_int(interp_degree), C.c_int(1 if fp64 else 0), P(u1), P(u11))
        return u1.reshape(nx, nx, nx), u11[: mesh.total]

    def renorm_density(self, nx, mesh, fdm, u1, u11):
        mh = abi.MeshHolder(mesh)
        u1 = np.ascontiguousarray(u1, np.float32).copy()
        u11 = np.ascontiguousarray(u11, np.float32).copy()
        if u11.shape[0] == 0:
            u11 = np.zeros((1, abi.NAMRX ** 3), np.float32)
        lib().orc_renorm_density(C.c_int(nx), C.byref(mh.c), C.c_float(fdm), P(u1), P(u11))
        return u1, u11[: mesh.total]

    def tsc_deposit(self, nx, lado0, dx, radx, rote, rete, mesh, fp64=True, parts=None):
        p = parts or self.p
        mh = abi.MeshHolder(mesh)
        u1 = np.zeros(nx ** 3, np.float32)
        u11 = np.zeros((max(mesh.total, 1), abi.NAMRX ** 3), np.float32)
        lib().orc_tsc_deposit(C.c_int(nx), C.c_float(lado0), C.c_float(dx), P(radx),
                              C.c_float(rote), C.c_float(rete), C.c_int64(p.n), P(p.x), P(p.y),
                              P(p.z), P(p.m), C.byref(mh.c), C.c_int(1 if fp64 else 0), P(u1),
                              P(u11))
        return u1.reshape(nx, nx, nx), u11[: mesh.total]

    def sort_x(self, nx, lado0):
        p = self.p
        nd = np.zeros(nx + 1, np.int32)
        lib().orc_sort_x(C.c_int64(p.n), *p.ptrs(), C.c_int(nx), C.c_float(lado0), P(nd, _ip))
        self.ndmpart_x = nd
        return nd

    def _store(self):
        p = self.p
        s = StoreC()
        s.n = p.n
        s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m, s.id = p.ptrs()
        s.ndmpart_x = P(self.ndmpart_x, _ip)
        s.norma = float(p.m.max())
        return s

    def prune_poor_haloes(self, consts, cat, low1, low2, facrad, do_need_to_count):
        s = self._store()
        cc = cat.as_c()
        lib().orc_prune_poor_haloes(C.byref(s), C.byref(consts), C.byref(cc), C.c_int(low1),
                                    C.c_int(low2), C.c_float(facrad), C.c_int(do_need_to_count))

    def check_rubish(self, cat, low1, low2):
        cc = cat.as_c()
        return lib().orc_check_rubish(C.byref(cc), C.c_int(cat.nclus), C.c_int(low1), C.c_int(low2))

    def accidental_substructure(self, cat):
        cc = cat.as_c()
        return lib().orc_accidental_substructure(C.byref(cc), C.c_int(cat.nclus))

    def halofind_grid_base(self, nx, dx, u1, radx, contrastec, rote, rete, rodo, re0, bound, vol_solap_low, cat,
                           mesh=None, u11=None):
        """HALOFIND_GRID at the base level (haloes_grids.f:287-582), with the
        recentering on the AMR levels when mesh and u11 are given: fills
        cat, returns NHALLEV(0)."""
        u = np.ascontiguousarray(u1, np.float32).reshape(-1)
        r = np.ascontiguousarray(radx, np.float32)
        cc = cat.as_c()
        mh = abi.MeshHolder(mesh) if mesh is not None else None
        v11 = np.ascontiguousarray(u11, np.float32).reshape(-1) if u11 is not None else None
        rc = lib().orc_halofind_grid_base(C.c_int(nx), C.c_float(dx), P(u), P(r), C.c_float(contrastec),
                                          C.c_float(rote), C.c_float(rete), C.c_float(rodo), C.c_float(re0),
                                          C.c_float(bound), C.c_float(vol_solap_low),
                                          C.byref(mh.c) if mh else None, P(v11) if v11 is not None else None,
                                          C.byref(cc))
        cat.nclus = cc.nclus
        if rc < 0:
            raise RuntimeError("HALOFIND_GRID: growing not converged" if rc == -1 else "catalogue full")
        return rc

    def halofind_grid_amr(self, ir, nx, dx, u1, radx, mesh, u11, cr0amr, cr0amr11, solap, contrastec, rote, rete,
                          rodo, re0, bound, vol_solap_low, cat):
        """HALOFIND_GRID on AMR level ir (haloes_grids.f:586-1097), appending to
        cat; returns NHALLEV(ir)."""
        f = lambda a, t=np.float32: np.ascontiguousarray(a, t).reshape(-1)
        u, r, v11 = f(u1), f(radx), f(u11)
        c0, c11, so = f(cr0amr, np.int32), f(cr0amr11, np.int32), f(solap, np.int32)
        mh = abi.MeshHolder(mesh)
        cc = cat.as_c()
        rc = lib().orc_halofind_grid_amr(C.c_int(ir), C.c_int(nx), C.c_float(dx), P(u), P(r), C.byref(mh.c), P(v11),
                                         P(c0, _ip), P(c11, _ip), P(so, _ip), C.c_float(contrastec),
                                         C.c_float(rote), C.c_float(rete), C.c_float(rodo), C.c_float(re0),
                                         C.c_float(bound), C.c_float(vol_solap_low), C.byref(cc))
        cat.nclus = cc.nclus
        if rc < 0:
            raise RuntimeError("HALOFIND_GRID: growing not converged" if rc == -1 else "catalogue full")
        return rc

    def search_substructure_grid(self, ir, nx, dx, u1, radx, mesh, u11, cr0amr, cr0amr11, solap, contrastec, rote,
                                 rete, rodo, re0, um, subs_lev, cat):
        """SEARCH_SUBSTRUCTURE_GRID on level ir (substructure.f:2-697); subs_lev
        (int32, NL+1 entries) is updated in place; returns SUBS_LEV(ir)."""
        f = lambda a, t=np.float32: np.ascontiguousarray(a, t).reshape(-1)
        u, r, v11 = f(u1), f(radx), f(u11)
        c0, c11, so = f(cr0amr, np.int32), f(cr0amr11, np.int32), f(solap, np.int32)
        assert subs_lev.dtype == np.int32 and subs_lev.flags.c_contiguous
        mh = abi.MeshHolder(mesh)
        cc = cat.as_c()
        rc = lib().orc_search_substructure_grid(C.c_int(ir), C.c_int(nx), C.c_float(dx), P(u), P(r), C.byref(mh.c),
                                                P(v11), P(c0, _ip), P(c11, _ip), P(so, _ip), C.c_float(contrastec),
                                                C.c_float(rote), C.c_float(rete), C.c_float(rodo), C.c_float(re0),
                                                C.c_float(um), P(subs_lev, _ip), C.byref(cc))
        cat.nclus = cc.nclus
        if rc < 0:
            raise RuntimeError({-2: "catalogue full", -3: "growth counts no cell"}.get(rc, str(rc)))
        return rc

    def overlapping(self, cat, ir, nhallev, vol_solap_low):
        """OVERLAPPING at level ir; nhallev[l] = haloes found at level l."""
        lowh3 = int(sum(nhallev[:ir])) + 1
        lowh2 = int(sum(nhallev[:ir + 1]))
        cc = cat.as_c()
        return lib().orc_overlapping(C.byref(cc), C.c_int(lowh3), C.c_int(lowh2), C.c_float(vol_solap_low))

    def halofind_particles(self, consts, mesh, cat, low1, low2, pph):
        s = self._store()
        cc = cat.as_c()
        mh = abi.MeshHolder(mesh)
        n = C.c_int64()
        rc = lib().orc_halofind_particles(C.byref(s), C.byref(consts), C.byref(mh.c),
                                          C.byref(cc), C.c_int(low1), C.c_int(low2),
                                          P(pph, _ip), C.c_int64(pph.shape[0]), C.byref(n),
                                          C.c_int(self.nthreads))
        if rc:
            raise RuntimeError(abi.ERRORS[rc])
        return n.value

    def substructure_particles(self, consts, mesh, cat, ir, subs_lev, pph):
        s = self._store()
        cc = cat.as_c()
        mh = abi.MeshHolder(mesh)
        n = C.c_int64()
        sl = np.ascontiguousarray(subs_lev, np.int32)
        rc = lib().orc_substructure_particles(C.byref(s), C.byref(consts), C.byref(mh.c),
                                              C.byref(cc), C.c_int(ir), P(sl, _ip),
                                              P(pph, _ip), C.c_int64(pph.shape[0]),
                                              C.byref(n), C.c_int(self.nthreads))
        if rc:
            raise RuntimeError(abi.ERRORS[rc])
        return n.value

    def mesh_base_counts(self, nx, dx, refine_thr, bor, npart_esp):
        """CREATE_MESH base-grid counts CR0 (grids.f:94-143), flat, IX fastest."""
        p = self.p
        esp = np.zeros(abi.N_ESP, np.int32)
        esp[:len(npart_esp)] = npart_esp
        out = np.empty(nx ** 3, np.int32)
        lib().orc_mesh_base_counts(C.c_int64(p.n), P(p.x), P(p.y), P(p.z), C.c_int(nx), C.c_float(dx),
                                   C.c_int(refine_thr), C.c_int(bor), P(esp, _ip), P(out, _ip))
        return out

    def mesh_patch_counts(self, irpa, dx, refine_thr, boramr, npart_esp, pnx, pny, pnz, prx, pry, prz):
        """CREATE_MESH counts on the patches of level irpa (grids.f:341-380)."""
        p = self.p
        esp = np.zeros(abi.N_ESP, np.int32)
        esp[:len(npart_esp)] = npart_esp
        ai = [np.ascontiguousarray(a, np.int32) for a in (pnx, pny, pnz)]
        af = [np.ascontiguousarray(a, np.float32) for a in (prx, pry, prz)]
        npatch = ai[0].shape[0]
        out = np.empty((npatch, abi.NAMRX ** 3), np.int32)
        lib().orc_mesh_patch_counts(C.c_int64(p.n), P(p.x), P(p.y), P(p.z), C.c_int(irpa), C.c_float(dx),
                                    C.c_int(refine_thr), C.c_int(boramr), P(esp, _ip), C.c_int(npatch),
                                    *[P(a, _ip) for a in ai], *[P(a) for a in af], P(out, _ip))
        return out

    def compute_cr0amr(self, nx, lado0, mesh):
        """COMPUTE_CR0AMR (grids.f:2076-2226): (CR0AMR nx^3, CR0AMR1 per patch)."""
        mh = abi.MeshHolder(mesh)
        ntot = int(np.asarray(mesh.npatch).sum())
        c0 = np.empty(nx ** 3, np.int32)
        c1 = np.empty((max(ntot, 1), abi.NAMRX ** 3), np.int32)
        lib().orc_compute_cr0amr(C.c_int(nx), C.c_float(lado0), C.byref(mh.c), P(c0, _ip), P(c1, _ip))
        return c0, c1[:ntot]

    def veinsgrid(self, ir, dx, radx1, mesh, solap):
        """VEINSGRID (grids.f:2229-2500) on level ir; solap ((npatch total,
        NAMRX^3) int32) written for the level's patches."""
        mh = abi.MeshHolder(mesh)
        assert solap.dtype == np.int32 and solap.flags.c_contiguous
        lib().orc_veinsgrid(C.c_int(ir), C.c_float(dx), C.c_float(radx1), C.byref(mh.c), P(solap, _ip))

    def veinsgrid_reduced(self, ir, dx, radx1, pnx, pny, pnz, prx, pry, prz, max_nb, cr01, conta11=None):
        """VEINSGRID_REDUCED (grids.f:1771-2073) on one level's patches; cr01
        and conta11 ((npatch, NAMRX^3) int32) are modified in place."""
        ai = [np.ascontiguousarray(a, np.int32) for a in (pnx, pny, pnz)]
        af = [np.ascontiguousarray(a, np.float32) for a in (prx, pry, prz)]
        assert cr01.dtype == np.int32 and cr01.flags.c_contiguous
        rc = lib().orc_veinsgrid_reduced(C.c_int(ir), C.c_float(dx), C.c_float(radx1), C.c_int(ai[0].shape[0]),
                                         *[P(a, _ip) for a in ai], *[P(a) for a in af], C.c_int(max_nb),
                                         P(cr01, _ip), P(conta11, _ip) if conta11 is not None else None)
        if rc:
            raise RuntimeError("VEINSGRID_REDUCED: too many neighbours" if rc == -1 else "out of memory")

    def poisson_fft(self, u1, dx):
        return poisson_fft(u1, dx)

    def final_ids(self, pph, n):
        return pph[:n].copy()
