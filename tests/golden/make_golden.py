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
    return out


if __name__ == "__main__":
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "tiny_oracle.npz"), **make())
    print("wrote tests/golden/tiny_oracle.npz")
