"""ctypes mirrors of include/asohf_types.h and numpy holders for them.

The layouts follow the Fortran driver's declarations (asohf.f:47-107): halo
arrays are SoA of length MAXNCLUS, ANGULARM(3,.), EIGENVAL(3,.),
INERTIA_TENSOR(6,.), PROFILES(NBINS,2,.) and INDCS_PARTICLES_PER_HALO(2,.)
are column-major, so halo i (0-based) owns a contiguous row.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

NAMRX = 32
NBINS = 20
NLEVELS = 9
N_ESP = 9

ERRORS = {
    0: "ok",
    1: "invalid argument",
    2: "CUDA error",
    3: "capacity exceeded",
    4: "device wait timed out",
    5: "NOT PRE-FOUND VIRIAL RADIUS",
    6: "wrong sorting, cannot continue",
    7: "no usable CUDA device",
    8: "unsupported option",
    9: "growing not converged",
}

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class MeshC(C.Structure):
    _fields_ = [("nl", C.c_int32), ("npatch", _ip),
                ("patchnx", _ip), ("patchny", _ip), ("patchnz", _ip),
                ("patchx", _ip), ("patchy", _ip), ("patchz", _ip),
                ("patchrx", _fp), ("patchry", _fp), ("patchrz", _fp),
                ("pare", _ip)]


class ParticlesC(C.Structure):
    _fields_ = [("n", C.c_int64), ("x", _fp), ("y", _fp), ("z", _fp),
                ("vx", _fp), ("vy", _fp), ("vz", _fp), ("m", _fp), ("id", _ip)]


class ConstsC(C.Structure):
    _fields_ = [("nx", C.c_int32), ("lado0", C.c_float), ("dx", C.c_float),
                ("rote", C.c_float), ("rete", C.c_float), ("pi", C.c_float),
                ("cgr", C.c_float), ("um", C.c_float), ("uv", C.c_float),
                ("contrastec", C.c_float), ("omegaz", C.c_float), ("fdm", C.c_float),
                ("zeta", C.c_float), ("min_num_part", C.c_int32),
                ("do_compute_energies", C.c_int32), ("max_part_dsum", C.c_int32),
                ("flag_wdm", C.c_int32), ("var", C.c_int32)]


CAT_FLOAT1 = ["masa", "radio", "clusrx", "clusry", "clusrz", "clusrxcm", "clusrycm",
              "clusrzcm", "msub", "rsub"]
CAT_INT1 = ["patchclus", "realclus", "levhal", "dmpclus"]
CAT_TAIL_FLOAT = ["vx", "vy", "vz", "mean_vr", "vcmax", "mcmax", "rcmax",
                  "m200c", "r200c", "m500c", "r500c", "m2500c", "r2500c",
                  "m200m", "r200m", "m500m", "r500m", "m2500m", "r2500m"]
CAT_SCALAR_FLOAT = (CAT_FLOAT1 + ["concentra", "vmaxclus"] + CAT_TAIL_FLOAT
                    + ["velocity_dispersion", "kinetic_e", "potential_e"])
CAT_SCALAR_INT = CAT_INT1 + ["iplip"]
CAT_MULTI = {"angularm": 3, "profiles": 2 * NBINS, "indcs": 2, "eigenval": 3,
             "inertia_tensor": 6}


class CatalogueC(C.Structure):
    _fields_ = ([("nclus", C.c_int32), ("capacity", C.c_int32)]
                + [(f, _fp) for f in CAT_FLOAT1]
                + [(f, _ip) for f in CAT_INT1]
                + [("concentra", _fp), ("angularm", _fp), ("vmaxclus", _fp),
                   ("iplip", _ip)]
                + [(f, _fp) for f in CAT_TAIL_FLOAT]
                + [("profiles", _fp), ("velocity_dispersion", _fp), ("kinetic_e", _fp),
                   ("potential_e", _fp), ("indcs", _ip), ("eigenval", _fp),
                   ("inertia_tensor", _fp)])


def _ptr(a: np.ndarray, t):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(t)


class Catalogue:
    """Host catalogue with the driver's initial values (INIT_OUTVARS,
    alloc.f:2-193: zeros everywhere)."""

    def __init__(self, capacity: int, pinned: bool = False):
        """pinned: arrays in page-locked host memory (torch), so the library's
        host<->device copies of the catalogue run at full PCIe speed."""
        self.capacity = int(capacity)
        self.nclus = 0
        self._keep = []

        def zeros(shape, dt):
            if not pinned:
                return np.zeros(shape, dt)
            import torch
            t = torch.zeros(shape, dtype=torch.int32 if dt == np.int32 else torch.float32).pin_memory()
            self._keep.append(t)
            return t.numpy()

        for f in CAT_SCALAR_FLOAT:
            setattr(self, f, zeros(capacity, np.float32))
        for f in CAT_SCALAR_INT:
            setattr(self, f, zeros(capacity, np.int32))
        for f, w in CAT_MULTI.items():
            dt = np.int32 if f == "indcs" else np.float32
            setattr(self, f, zeros((capacity, w), dt))

    def fields(self):
        return CAT_SCALAR_FLOAT + CAT_SCALAR_INT + list(CAT_MULTI)

    def reset(self):
        """Back to the initial state (zeros, nclus = 0).  Entries past nclus
        are never written, so only the first nclus are cleared."""
        n = self.nclus
        if n:
            for f in self.fields():
                getattr(self, f)[:n] = 0
        self.nclus = 0
        return self

    def copy(self) -> "Catalogue":
        c = Catalogue.__new__(Catalogue)
        c.capacity, c.nclus = self.capacity, self.nclus
        c._keep = []
        for f in self.fields():
            setattr(c, f, getattr(self, f).copy())
        return c

    def as_c(self) -> CatalogueC:
        s = CatalogueC()
        s.nclus, s.capacity = self.nclus, self.capacity
        for name, t in CatalogueC._fields_[2:]:
            setattr(s, name, _ptr(getattr(self, name), t))
        return s


class MeshHolder:
    """Keeps the int32/float32 arrays of a synth.Mesh alive for a MeshC."""

    def __init__(self, mesh):
        self.arrays = {}
        for f in ["npatch", "patchnx", "patchny", "patchnz", "patchx", "patchy", "patchz",
                  "pare"]:
            self.arrays[f] = np.ascontiguousarray(getattr(mesh, f), np.int32)
        for f in ["patchrx", "patchry", "patchrz"]:
            self.arrays[f] = np.ascontiguousarray(getattr(mesh, f), np.float32)
        self.c = MeshC()
        self.c.nl = int(mesh.nl)
        for name, t in MeshC._fields_[1:]:
            setattr(self.c, name, _ptr(self.arrays[name], t))


def consts_c(nx, lado0, dx, cos, fdm, zeta, min_num_part, do_compute_energies=0,
             max_part_dsum=4000, flag_wdm=1, var=1) -> ConstsC:
    k = ConstsC()
    k.nx, k.lado0, k.dx = nx, lado0, dx
    k.rote, k.rete, k.pi, k.cgr = cos["rote"], cos["rete"], cos["pi"], cos["cgr"]
    k.um, k.uv = cos["um"], cos["uv"]
    k.contrastec, k.omegaz = cos["contrastec"], cos["omegaz"]
    k.fdm, k.zeta = fdm, zeta
    k.min_num_part, k.do_compute_energies = min_num_part, do_compute_energies
    k.max_part_dsum, k.flag_wdm, k.var = max_part_dsum, flag_wdm, var
    return k
