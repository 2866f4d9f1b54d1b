"""Catalogue comparison shared by the GPU parity tests: integer fields and
the ID stream identical, float fields within a relative tolerance (1e-5:
the device sums in float64 in a different order than the sequential
Fortran loops)."""
import numpy as np

INT_FIELDS = ["realclus", "dmpclus", "indcs", "iplip"]
FLOAT_FIELDS = ["masa", "radio", "clusrx", "clusry", "clusrz", "clusrxcm", "clusrycm", "clusrzcm",
                "vx", "vy", "vz", "mean_vr", "vcmax", "mcmax", "rcmax", "m200c", "r200c", "m500c",
                "r500c", "m2500c", "r2500c", "m200m", "r200m", "m500m", "r500m", "m2500m", "r2500m",
                "velocity_dispersion", "vmaxclus", "angularm", "inertia_tensor", "eigenval", "profiles",
                "msub", "rsub"]


def compare(rg, ro, rtol=1e-5):
    n = ro.cat.nclus
    assert rg.cat.nclus == n
    for f in INT_FIELDS:
        a, b = getattr(rg.cat, f)[:n], getattr(ro.cat, f)[:n]
        assert np.array_equal(a, b), (f, np.nonzero(a != b))
    bad = {}
    for f in FLOAT_FIELDS:
        a = getattr(rg.cat, f)[:n].astype(np.float64)
        b = getattr(ro.cat, f)[:n].astype(np.float64)
        tol = rtol * np.maximum(np.abs(b), 1e-30) + 1e-30
        if f in ("mean_vr", "angularm", "vx", "vy", "vz", "inertia_tensor"):
            # sums of signed terms: compare against the field's scale
            tol = rtol * max(np.abs(b).max(), 1e-30) + 0 * tol
        nbad = int(np.count_nonzero(np.abs(a - b) > tol))
        if nbad:
            bad[f] = nbad
    assert not bad, bad
    assert np.array_equal(rg.pph, ro.pph)
