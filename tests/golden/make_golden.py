"""Generates the golden vectors of the CPU oracle on the 32^3-particle test
snapshot (tests/golden/tiny_oracle.npz).  The reference cannot be built here
(no Fortran compiler), so these vectors pin the oracle against change; they
are not reference outputs.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from asohf_b200 import driver, synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

SCALARS = ["masa", "radio", "clusrx", "clusry", "clusrz", "clusrxcm", "clusrycm", "clusrzcm", "msub",
           "rsub", "realclus", "dmpclus", "iplip", "vx", "vy", "vz", "m200c", "r200c", "m200m", "r200m",
           "vcmax", "velocity_dispersion"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make():
    s = synth.generate("tiny")
    r = driver.run(s, O.OracleBackend(nthreads=1), with_subs=True)
    n = r.cat.nclus
    out = {"npart_esp": r.npart_esp, "ndmpart_x": r.ndmpart_x, "nclus": np.array([n]),
           "subs_lev": r.subs_lev, "pph": r.pph,
           "u1_sha256": np.array([digest(r.u1)]), "u11_sha256": np.array([digest(r.u11)]),
           "u1_sample": r.u1.ravel()[::97].copy(), "indcs": r.cat.indcs[:n].copy()}
    for f in SCALARS:
        out["cat_" + f] = getattr(r.cat, f)[:n].copy()
    out.update(make_mesh_and_grid_finder(s, r))
    return out


def make_mesh_and_grid_finder(s, r):
    """The mesh builder's counts and VEINSGRID_REDUCED on the snapshot's
    level-1 patches, and the base level of the grid finder on its density."""
    from asohf_b200 import abi
    cfg = s.cfg
    plan = driver.prepare(s)
    dx = float(plan.dx)
    ob = O.OracleBackend(nthreads=1)
    ob.upload(s)
    npe = ob.species_sort(cfg.nx, plan.dx, plan.cos["rodo"], plan.cos["re0"])
    cr0 = ob.mesh_base_counts(cfg.nx, dx, 8, 2, npe)
    m = plan.mesh
    n1 = int(m.npatch[1])
    pat = (m.patchnx[:n1], m.patchny[:n1], m.patchnz[:n1], m.patchrx[:n1], m.patchry[:n1], m.patchrz[:n1])
    cr01 = ob.mesh_patch_counts(1, dx, 8, 1, npe, *pat)
    ob.veinsgrid_reduced(1, dx, float(plan.radx[1]), *pat, 1000, cr01)
    cat = abi.Catalogue(4096)
    nh = ob.halofind_grid_base(cfg.nx, dx, r.u1, plan.radx, 200.0, 1.0, 1.0, 1.0, 1.0, 10.0 * dx, 0.2, cat,
                               mesh=m, u11=r.u11)
    # the whole grid finder on the level-1 mesh: masks, base level, level 1
    m1 = synth.Mesh(1, np.array([0, n1], np.int32), *(np.ascontiguousarray(a[:n1]) for a in (
        m.patchnx, m.patchny, m.patchnz, m.patchx, m.patchy, m.patchz, m.patchrx, m.patchry, m.patchrz)),
        np.zeros(n1, np.int32))
    c0, c11 = ob.compute_cr0amr(cfg.nx, float(cfg.lado0), m1)
    so = np.zeros((n1, abi.NAMRX ** 3), np.int32)
    ob.veinsgrid(1, dx, float(plan.radx[1]), m1, so)
    u11_1 = np.ascontiguousarray(r.u11[:n1])
    g = abi.Catalogue(4096)
    n0 = ob.halofind_grid_base(cfg.nx, dx, r.u1, plan.radx, 200.0, 1.0, 1.0, 1.0, 1.0, 10.0 * dx, 0.2, g,
                               mesh=m1, u11=u11_1)
    na1 = ob.halofind_grid_amr(1, cfg.nx, dx, r.u1, plan.radx, m1, u11_1, c0, c11, so, 200.0, 1.0, 1.0, 1.0, 1.0,
                               10.0 * dx, 0.2, g)
    k = g.nclus
    # subhalo seeding on level 1 inside the haloes of the particle pipeline's catalogue
    sc = abi.Catalogue(r.cat.capacity + 4096)
    nh = int(r.subs_lev[0]) if len(r.subs_lev) else r.cat.nclus
    sc.nclus = nh
    for f in ("realclus", "levhal", "clusrx", "clusry", "clusrz", "radio", "rsub", "masa", "msub", "profiles"):
        getattr(sc, f)[:nh] = getattr(r.cat, f)[:nh]
    sl = np.zeros(2, np.int32)
    sl[0] = nh
    ns = ob.search_substructure_grid(1, cfg.nx, dx, r.u1, plan.radx, m1, u11_1, c0, c11, so, 200.0, 1.0, 1.0, 1.0,
                                     1.0, 1.0, sl, sc)
    sub = {"gridsub_n": np.array([ns]), "gridsub_realclus": sc.realclus[nh:sc.nclus].copy(),
           "gridsub_rsub": sc.rsub[nh:sc.nclus].copy(), "gridsub_clusrx": sc.clusrx[nh:sc.nclus].copy()}
    amr = {**sub, "gridamr_cr0amr_sha256": np.array([digest(c0)]), "gridamr_solap_sha256": np.array([digest(so)]),
           "gridamr_nhallev": np.array([n0, na1]), "gridamr_levhal": g.levhal[:k].copy(),
           "gridamr_realclus": g.realclus[:k].copy(), "gridamr_radio": g.radio[:k].copy(),
           "gridamr_clusrx": g.clusrx[:k].copy(), "gridamr_patchclus": g.patchclus[:k].copy()}
    return {**amr, "mesh_cr0_sha256": np.array([digest(cr0)]), "mesh_cr01_sha256": np.array([digest(cr01)]),
            "mesh_cr01_nonzero": np.array([int((cr01 > 0).sum())]),
            "grid_nhallev0": np.array([nh]), "grid_radio": cat.radio[:cat.nclus].copy(),
            "grid_clusrx": cat.clusrx[:cat.nclus].copy(), "grid_realclus": cat.realclus[:cat.nclus].copy()}


if __name__ == "__main__":
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "tiny_oracle.npz"), **make())
    print("wrote tests/golden/tiny_oracle.npz")
