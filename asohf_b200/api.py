"""Python binding of libasohf_gpu.so (ctypes) -- the host mirror of the
reference's subroutine interface for the particle hot path.

``Asohf`` owns one library context (device, CUDA stream, device particle
store).  Its methods are named after the reference subroutines they replace
and take numpy arrays (host: the library stages them) or torch CUDA tensors
(device: no copies).  There is no CPU fallback: without the built library or
a CUDA device every call raises.

``GpuBackend`` adapts ``Asohf`` to the method set the hot-path driver
(asohf_b200.driver) uses.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_LIB = None
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_vp = C.c_void_p


class AsohfError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        detail = ""
        if _LIB is not None and code == 2:
            detail = ": " + _LIB.asohf_last_error_detail().decode()
        super().__init__(f"{what}: {abi.ERRORS.get(code, 'status %d' % code)}{detail}")


def lib_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libasohf_gpu.so")


def load():
    """Loads libasohf_gpu.so; raises if it was not built."""
    global _LIB
    if _LIB is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m asohf_b200.build` "
                               "(the hot path has no CPU fallback)")
        L = C.CDLL(path)
        L.asohf_strerror.restype = C.c_char_p
        L.asohf_last_error_detail.restype = C.c_char_p
        L.asohf_launch_count.restype = C.c_int64
        L.asohf_launch_count.argtypes = [_vp]
        for name in ["asohf_create", "asohf_destroy", "asohf_set_stream", "asohf_synchronize",
                     "asohf_upload_particles", "asohf_download_particles",
                     "asohf_sort_dm_particles_localdensity", "asohf_density",
                     "asohf_renorm_density", "asohf_interpolate_density_tsc", "asohf_poisson_fft",
                     "asohf_tsc_poisson_forward", "asohf_tsc_poisson_adjoint",
                     "asohf_sort_dm_particles_x", "asohf_prune_poor_haloes",
                     "asohf_halofind_particles", "asohf_substructure_particles",
                     "asohf_get_particles_per_halo", "asohf_set_profiling", "asohf_kernel_stats",
                     "asohf_work_counters", "asohf_set_cluster_threshold", "asohf_set_group_tiers",
                     "asohf_copy_to_host_sm", "asohf_set_cluster_share", "asohf_prefetch_particles",
                     "asohf_copy_to_host_async", "asohf_copy_wait",
                     "asohf_check_rubish", "asohf_accidental_substructure", "asohf_re_sort_haloes"]:
            getattr(L, name).restype = C.c_int
        _LIB = L
    return _LIB


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    """Pointer of a numpy array or torch tensor (contiguous)."""
    if a is None:
        return None
    if _is_torch(a):
        assert a.is_contiguous()
        return C.c_void_p(a.data_ptr())
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _check(rc: int, what: str):
    if rc != 0:
        raise AsohfError(rc, what)


class Asohf:
    """One library context on one CUDA device."""

    def __init__(self, device: int = 0):
        self.L = load()
        self.h = C.c_void_p()
        _check(self.L.asohf_create(C.c_int(device), C.byref(self.h)), "asohf_create")
        self.device = device
        self.n = 0

    def close(self):
        if self.h:
            self.L.asohf_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        _check(self.L.asohf_set_stream(self.h, C.c_void_p(stream_ptr)), "asohf_set_stream")

    def synchronize(self):
        _check(self.L.asohf_synchronize(self.h), "asohf_synchronize")

    def launch_count(self) -> int:
        return int(self.L.asohf_launch_count(self.h))

    def set_density_overlap(self, on: bool):
        """Deferred AMR-patch deposit for device outputs (see
        asohf_set_density_overlap); U11 is complete after density_wait."""
        _check(self.L.asohf_set_density_overlap(self.h, C.c_int(int(on))), "asohf_set_density_overlap")

    def density_wait(self, stream_ptr: int):
        """Makes the CUDA stream `stream_ptr` wait for a deferred patch deposit."""
        _check(self.L.asohf_density_wait(self.h, C.c_void_p(stream_ptr)), "asohf_density_wait")

    def set_epot_seed(self, seed: int):
        """Seed of COMPUTE_EPOT's sampling estimator (default 1)."""
        _check(self.L.asohf_set_epot_seed(self.h, C.c_uint32(int(seed))), "asohf_set_epot_seed")

    def set_cluster_threshold(self, min_members: int):
        """Haloes with at least min_members members go to the cluster path
        (0: default)."""
        _check(self.L.asohf_set_cluster_threshold(self.h, C.c_int64(int(min_members))),
               "asohf_set_cluster_threshold")

    def set_cluster_share(self, members_per_cta: int):
        """Entries per CTA from which the halo kernel widens its clusters (0: default)."""
        _check(self.L.asohf_set_cluster_share(self.h, C.c_int64(int(members_per_cta))), "asohf_set_cluster_share")

    def set_group_tiers(self, tier1: int, tier2: int):
        """Member counts from which a halo gets 128 / 256 threads (0: default)."""
        _check(self.L.asohf_set_group_tiers(self.h, C.c_int64(int(tier1)), C.c_int64(int(tier2))),
               "asohf_set_group_tiers")

    def set_profiling(self, on: bool):
        """Brackets the main kernels with CUDA events (diagnostics)."""
        _check(self.L.asohf_set_profiling(self.h, C.c_int(int(on))), "asohf_set_profiling")

    def copy_to_host_sm(self, dst, src, stream=None):
        """Enqueues dst[:] = src[:] (page-locked host tensor <- device tensor
        of this context's GPU, same byte size, a multiple of 16) as SM
        stores on `stream` (a torch stream; the context stream when None)."""
        import torch
        nb = src.numel() * src.element_size()
        if not dst.is_pinned() or dst.numel() * dst.element_size() != nb or not dst.is_contiguous() \
                or not src.is_contiguous() or not src.is_cuda or dst.dtype != src.dtype:
            raise ValueError("copy_to_host_sm: a contiguous page-locked tensor of the device tensor's size")
        s = C.c_void_p(stream.cuda_stream if stream is not None else 0)
        head = nb - nb % 16 if dst.data_ptr() % 16 == 0 and src.data_ptr() % 16 == 0 else 0
        _check(self.L.asohf_copy_to_host_sm(self.h, C.c_void_p(dst.data_ptr()), C.c_void_p(src.data_ptr()),
                                            C.c_int64(head), s), "asohf_copy_to_host_sm")
        if head < nb:  # the last few bytes (or an unaligned buffer) by an ordinary copy on the same stream
            e = head // src.element_size()
            with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
                dst.view(-1)[e:].copy_(src.view(-1)[e:], non_blocking=True)

    def work_counters(self, reset: bool = False):
        """Element-passes of the halo (entry 0) and subhalo (entry 1) kernels."""
        out = np.zeros(8, np.int64)
        _check(self.L.asohf_work_counters(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)), C.c_int(int(reset))),
               "asohf_work_counters")
        return out

    def kernel_stats(self) -> dict:
        """{kernel name: (total device ms, launches)} since profiling was enabled."""
        out = {}
        i = 0
        while True:
            name = C.c_char_p()
            ms = C.c_double()
            n = C.c_int64()
            if self.L.asohf_kernel_stats(self.h, C.c_int(i), C.byref(name), C.byref(ms), C.byref(n)) != 0:
                break
            out[name.value.decode()] = (ms.value, n.value)
            i += 1
        return out

    # -------------------------------------------------------------- particles
    def upload_particles(self, x, y, z, vx, vy, vz, m, ids):
        dev = _is_torch(x) and x.is_cuda
        p = abi.ParticlesC()
        p.n = int(x.shape[0])
        for f, a in zip(["x", "y", "z", "vx", "vy", "vz", "m"], [x, y, z, vx, vy, vz, m]):
            setattr(p, f, C.cast(_ptr(a), _fp))
        p.id = C.cast(_ptr(ids), _ip)
        _check(self.L.asohf_upload_particles(self.h, C.byref(p), C.c_int(int(dev))),
               "asohf_upload_particles")
        self.n = p.n

    def copy_to_host_async(self, dst, src):
        """Copy of device tensor src into page-locked host tensor dst (same
        size) on a copy engine, chunk by chunk, after the work issued so far;
        copy_wait() waits for every such copy."""
        if dst.numel() * dst.element_size() != src.numel() * src.element_size() or not dst.is_pinned():
            raise ValueError("copy_to_host_async: a page-locked tensor of the device tensor's size")
        _check(self.L.asohf_copy_to_host_async(self.h, C.c_void_p(dst.data_ptr()), C.c_void_p(src.data_ptr()),
                                               C.c_int64(src.numel() * src.element_size())),
               "asohf_copy_to_host_async")

    def copy_wait(self, stream=None):
        """Makes `stream` (the host, when None) wait for the copies of
        copy_to_host_async issued so far."""
        s = C.c_void_p(stream.cuda_stream) if stream is not None else None
        _check(self.L.asohf_copy_wait(self.h, s), "asohf_copy_wait")

    def prefetch_particles(self, x, y, z, vx, vy, vz, m, ids):
        """Starts copying these host arrays (page-locked) for the next
        upload_particles of the same arrays, beside the work in flight."""
        p = abi.ParticlesC()
        p.n = int(x.shape[0])
        for f, a in zip(["x", "y", "z", "vx", "vy", "vz", "m"], [x, y, z, vx, vy, vz, m]):
            setattr(p, f, C.cast(_ptr(a), _fp))
        p.id = C.cast(_ptr(ids), _ip)
        _check(self.L.asohf_prefetch_particles(self.h, C.byref(p)), "asohf_prefetch_particles")

    def download_particles(self, out=None):
        """Returns (x, y, z, vx, vy, vz, m, id) numpy arrays in store order."""
        n = self.n
        if out is None:
            out = [np.empty(n, np.float32) for _ in range(7)] + [np.empty(n, np.int32)]
        p = abi.ParticlesC()
        p.n = n
        for f, a in zip(["x", "y", "z", "vx", "vy", "vz", "m"], out[:7]):
            setattr(p, f, C.cast(_ptr(a), _fp))
        p.id = C.cast(_ptr(out[7]), _ip)
        dev = _is_torch(out[0])
        _check(self.L.asohf_download_particles(self.h, C.byref(p), C.c_int(int(dev))),
               "asohf_download_particles")
        return out

    # -------------------------------------------------------------- mesh stage
    def sort_dm_particles_localdensity(self, nx, dx, rodo, re0):
        """SORT_DM_PARTICLES_LOCALDENSITY (reader.f:140-336)."""
        npe = np.zeros(abi.N_ESP, np.int32)
        _check(self.L.asohf_sort_dm_particles_localdensity(
            self.h, C.c_int(nx), C.c_float(dx), C.c_float(rodo), C.c_float(re0),
            npe.ctypes.data_as(_ip)), "SORT_DM_PARTICLES_LOCALDENSITY")
        return npe

    def density(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, u1, u11):
        """DENSITY (grids.f:710-994) into u1 (NX^3) and u11 (P x 32^3)."""
        mh = abi.MeshHolder(mesh)
        dev = _is_torch(u1)
        npe = np.ascontiguousarray(npart_esp, np.int32)
        _check(self.L.asohf_density(self.h, C.c_int(nx), C.c_float(lado0), C.c_float(dx),
                                    C.c_float(rote), C.c_float(rete), npe.ctypes.data_as(_ip),
                                    C.byref(mh.c), C.c_int(interp_degree), _ptr(u1), _ptr(u11),
                                    C.c_int(int(dev))), "DENSITY")

    def renorm_density(self, nx, mesh, fdm, u1, u11):
        """RENORM_DENSITY (grids.f:2668-2722), in place."""
        mh = abi.MeshHolder(mesh)
        _check(self.L.asohf_renorm_density(self.h, C.c_int(nx), C.byref(mh.c), C.c_float(fdm),
                                           _ptr(u1), _ptr(u11), C.c_int(int(_is_torch(u1)))),
               "RENORM_DENSITY")

    def interpolate_density_tsc(self, nx, lado0, dx, radx, rote, rete, mesh, u1, u11):
        """INTERPOLATE_DENSITY_TSC (grids.f:1070-1398)."""
        mh = abi.MeshHolder(mesh)
        r = np.ascontiguousarray(radx, np.float32)
        _check(self.L.asohf_interpolate_density_tsc(
            self.h, C.c_int(nx), C.c_float(lado0), C.c_float(dx), r.ctypes.data_as(_fp),
            C.c_float(rote), C.c_float(rete), C.byref(mh.c), _ptr(u1), _ptr(u11),
            C.c_int(int(_is_torch(u1)))), "INTERPOLATE_DENSITY_TSC")

    def mesh_base_counts(self, nx, dx, refine_thr, bor, npart_esp, out=None):
        """CREATE_MESH base-grid counts CR0 (grids.f:107-143), flat nx^3, IX fastest."""
        esp = np.zeros(abi.N_ESP, np.int32)
        esp[:len(npart_esp)] = npart_esp
        if out is None:
            out = np.empty(nx ** 3, np.int32)
        _check(self.L.asohf_mesh_base_counts(self.h, C.c_int(nx), C.c_float(dx), C.c_int(refine_thr), C.c_int(bor),
                                             esp.ctypes.data_as(C.c_void_p), _ptr(out),
                                             C.c_int(int(_is_torch(out)))), "CREATE_MESH counts")
        return out

    def mesh_patch_counts(self, nx, lado0, dx, irpa, refine_thr, boramr, npart_esp, pnx, pny, pnz, prx, pry, prz,
                          out=None):
        """CREATE_MESH counts CR01 on the patches of level irpa (grids.f:341-380),
        (npatch, NAMRX^3) int32, IX fastest."""
        esp = np.zeros(abi.N_ESP, np.int32)
        esp[:len(npart_esp)] = npart_esp
        ai = [np.ascontiguousarray(a, np.int32) for a in (pnx, pny, pnz)]
        af = [np.ascontiguousarray(a, np.float32) for a in (prx, pry, prz)]
        npatch = int(ai[0].shape[0])
        if out is None:
            out = np.empty((npatch, abi.NAMRX ** 3), np.int32)
        _check(self.L.asohf_mesh_patch_counts(
            self.h, C.c_int(nx), C.c_float(lado0), C.c_float(dx), C.c_int(irpa), C.c_int(refine_thr),
            C.c_int(boramr), esp.ctypes.data_as(C.c_void_p), C.c_int(npatch),
            *[a.ctypes.data_as(C.c_void_p) for a in ai], *[a.ctypes.data_as(C.c_void_p) for a in af],
            _ptr(out), C.c_int(int(_is_torch(out)))), "CREATE_MESH patch counts")
        return out

    def veinsgrid_reduced(self, ir, dx, radx1, pnx, pny, pnz, prx, pry, prz, max_neighbours, cr01, conta11=None):
        """VEINSGRID_REDUCED (grids.f:1771-2073) on one level's patches; cr01 and
        conta11 ((npatch, NAMRX^3) int32, numpy or CUDA tensors) in place."""
        ai = [np.ascontiguousarray(a, np.int32) for a in (pnx, pny, pnz)]
        af = [np.ascontiguousarray(a, np.float32) for a in (prx, pry, prz)]
        _check(self.L.asohf_veinsgrid_reduced(
            self.h, C.c_int(ir), C.c_float(dx), C.c_float(radx1), C.c_int(int(ai[0].shape[0])),
            *[a.ctypes.data_as(C.c_void_p) for a in ai], *[a.ctypes.data_as(C.c_void_p) for a in af],
            C.c_int(max_neighbours), _ptr(cr01), _ptr(conta11) if conta11 is not None else None,
            C.c_int(int(_is_torch(cr01)))), "VEINSGRID_REDUCED")

    def poisson_fft(self, nx, dx, rho, pot, batch=1):
        """MOMENTO + POFFT3D (poisson.f:98-249)."""
        _check(self.L.asohf_poisson_fft(self.h, C.c_int(nx), C.c_float(dx), C.c_int(batch),
                                        _ptr(rho), _ptr(pot), C.c_int(int(_is_torch(rho)))),
               "POFFT3D")

    def tsc_poisson_forward(self, nx, lado0, dx, radx, rote, rete, x, y, z, m, rho, pot, batch):
        r = np.ascontiguousarray(radx, np.float32)
        n_per = int(x.numel()) // batch
        _check(self.L.asohf_tsc_poisson_forward(
            self.h, C.c_int(nx), C.c_float(lado0), C.c_float(dx), r.ctypes.data_as(_fp),
            C.c_float(rote), C.c_float(rete), C.c_int(batch), C.c_int64(n_per), _ptr(x), _ptr(y),
            _ptr(z), _ptr(m), _ptr(rho), _ptr(pot)), "deposit+Poisson forward")

    def tsc_poisson_adjoint(self, nx, lado0, dx, radx, rote, rete, x, y, z, m, w, gx, gy, gz, gm,
                            batch):
        r = np.ascontiguousarray(radx, np.float32)
        n_per = int(x.numel()) // batch
        _check(self.L.asohf_tsc_poisson_adjoint(
            self.h, C.c_int(nx), C.c_float(lado0), C.c_float(dx), r.ctypes.data_as(_fp),
            C.c_float(rote), C.c_float(rete), C.c_int(batch), C.c_int64(n_per), _ptr(x), _ptr(y),
            _ptr(z), _ptr(m), _ptr(w), _ptr(gx), _ptr(gy), _ptr(gz), _ptr(gm)),
            "deposit+Poisson adjoint")

    # -------------------------------------------------------------- halo stage
    def sort_dm_particles_x(self, nx, lado0):
        """SORT_DM_PARTICLES_X (grids.f:2726-2838); returns NDMPART_X(0:NX)."""
        nd = np.zeros(nx + 1, np.int32)
        _check(self.L.asohf_sort_dm_particles_x(self.h, C.c_int(nx), C.c_float(lado0),
                                                nd.ctypes.data_as(_ip)), "SORT_DM_PARTICLES_X")
        return nd

    def prune_poor_haloes(self, consts, cat, low1, low2, facrad, do_need_to_count):
        cc = cat.as_c()
        _check(self.L.asohf_prune_poor_haloes(self.h, C.byref(consts), C.byref(cc), C.c_int(low1),
                                              C.c_int(low2), C.c_float(facrad),
                                              C.c_int(do_need_to_count), C.c_int(0)),
               "PRUNE_POOR_HALOES")

    def check_rubish(self, cat, low1, low2):
        """CHECK_RUBISH over the window low1..low2; returns KONTA."""
        cc = cat.as_c()
        n = C.c_int32()
        _check(self.L.asohf_check_rubish(self.h, C.byref(cc), C.c_int(cat.nclus), C.c_int(low1), C.c_int(low2),
                                         C.c_int(0), C.byref(n)), "CHECK_RUBISH")
        return n.value

    def accidental_substructure(self, cat):
        """ACCIDENTAL_SUBSTRUCTURE over the catalogue; returns KONTA."""
        cc = cat.as_c()
        n = C.c_int32()
        _check(self.L.asohf_accidental_substructure(self.h, C.byref(cc), C.c_int(cat.nclus), C.c_int(0),
                                                    C.byref(n)), "ACCIDENTAL_SUBSTRUCTURE")
        return n.value

    def re_sort_haloes(self, cat, nhallev, ir):
        """RE_SORT_HALOES (haloes_particles.f:2-56) on the host catalogue:
        drops the REALCLUS = 0 entries of level ir in order; nhallev[ir] and
        cat.nclus are updated; returns the window's keep mask."""
        nh = np.array(nhallev, np.int32)
        w = int(nh[ir])
        keep = np.zeros(max(w, 1), np.uint8)
        cc = cat.as_c()
        _check(self.L.asohf_re_sort_haloes(self.h, C.byref(cc), nh.ctypes.data_as(C.POINTER(C.c_int32)),
                                           C.c_int(ir), keep.ctypes.data_as(C.POINTER(C.c_uint8))),
               "RE_SORT_HALOES")
        nhallev[ir] = nh[ir]
        cat.nclus = cc.nclus
        return keep[:w].astype(bool) if w else np.zeros(0, bool)

    def overlapping(self, cat, ir, nhallev, vol_solap_low):
        """OVERLAPPING at level ir (nhallev[l]: haloes of level l); returns
        the number of removed haloes among level ir's."""
        nh = np.ascontiguousarray(nhallev[:ir + 1], dtype=np.int32)
        cc = cat.as_c()
        n = C.c_int32()
        _check(self.L.asohf_overlapping(self.h, C.byref(cc), C.c_int(ir), nh.ctypes.data_as(C.c_void_p),
                                        C.c_float(vol_solap_low), C.c_int(0), C.byref(n)), "OVERLAPPING")
        return n.value

    def halofind_grid_base(self, nx, dx, u1, radx, contrastec, rote, rete, rodo, re0, bound, vol_solap_low, cat):
        """HALOFIND_GRID at the base level without AMR recentering; u1 is a
        host array or a torch CUDA tensor; fills cat (host), returns
        NHALLEV(0)."""
        if _is_torch(u1) and u1.is_cuda:
            u, on_dev = u1.contiguous(), 1
        else:
            u, on_dev = np.ascontiguousarray(u1, np.float32).reshape(-1), 0
        r = np.ascontiguousarray(radx, np.float32)
        cc = cat.as_c()
        n = C.c_int32()
        f = C.c_float
        # the catalogue stays on the host: the grid is read in place on the device
        _check(self.L.asohf_halofind_grid_base(self.h, C.c_int(nx), f(dx), _ptr(u), _ptr(r), f(contrastec), f(rote),
                                               f(rete), f(rodo), f(re0), f(bound), f(vol_solap_low), None,
                                               C.byref(cc), C.c_int(on_dev), C.c_int(0), C.byref(n)),
               "HALOFIND_GRID")
        cat.nclus = cc.nclus
        return n.value

    def halofind_particles(self, consts, mesh, cat, low1, low2):
        mh = abi.MeshHolder(mesh)
        cc = cat.as_c()
        _check(self.L.asohf_halofind_particles(self.h, C.byref(consts), C.byref(mh.c), C.byref(cc),
                                               C.c_int(low1), C.c_int(low2), C.c_int(0)),
               "HALOFIND_PARTICLES")

    def substructure_particles(self, consts, mesh, cat, ir, subs_lev):
        mh = abi.MeshHolder(mesh)
        cc = cat.as_c()
        sl = np.ascontiguousarray(subs_lev, np.int32)
        _check(self.L.asohf_substructure_particles(self.h, C.byref(consts), C.byref(mh.c),
                                                   C.byref(cc), C.c_int(ir), sl.ctypes.data_as(_ip),
                                                   C.c_int(0)), "SUBSTRUCTURE_PARTICLES")

    def particles_per_halo(self, out=None):
        """The bound-particle ID stream.  out: None (a new numpy array), a
        host numpy array or a torch CUDA tensor of at least the stream's
        length; returns the filled prefix."""
        n = C.c_int64()
        _check(self.L.asohf_get_particles_per_halo(self.h, None, C.c_int64(0), C.byref(n), C.c_int(0)),
               "PARTICLES_PER_HALO")
        if out is None:
            out = np.zeros(max(n.value, 1), np.int32)
        on_dev = _is_torch(out) and out.is_cuda
        _check(self.L.asohf_get_particles_per_halo(self.h, C.cast(_ptr(out), _ip),
                                                   C.c_int64(out.shape[0]), C.byref(n), C.c_int(int(on_dev))),
               "PARTICLES_PER_HALO")
        return out[: n.value]


class GpuBackend:
    """Backend of asohf_b200.driver on the B200 library (host arrays)."""

    name = "gpu"

    pinned_host = True  # host catalogue in page-locked memory

    def __init__(self, device: int = 0, cluster_threshold: int = 0, tiers=(0, 0), cluster_share: int = 0):
        self.a = Asohf(device)
        self._ids = None
        # the patch deposit of density_renorm runs beside the x-sort and the
        # halo finder; the grid copies and sync_outputs wait for it
        self.a.set_density_overlap(True)
        if cluster_threshold:
            self.a.set_cluster_threshold(cluster_threshold)
        if cluster_share:
            self.a.set_cluster_share(cluster_share)
        if tiers != (0, 0):
            self.a.set_group_tiers(*tiers)

    # host particles of the next run, copied while this run computes (set by
    # a caller that runs snapshots back to back; None: no prefetch)
    prefetch_next = None

    def prefetch(self, parts):
        self.a.prefetch_particles(parts.x, parts.y, parts.z, parts.vx, parts.vy, parts.vz, parts.m, parts.id)

    def upload(self, parts):
        self.a.upload_particles(parts.x, parts.y, parts.z, parts.vx, parts.vy, parts.vz, parts.m,
                                parts.id)
        if self.prefetch_next is not None:
            self.prefetch(self.prefetch_next)

    def download(self):
        from types import SimpleNamespace
        x, y, z, vx, vy, vz, m, i = self.a.download_particles()
        return SimpleNamespace(x=x, y=y, z=z, vx=vx, vy=vy, vz=vz, m=m, id=i, n=x.shape[0])

    def species_sort(self, nx, dx, rodo, re0):
        return self.a.sort_dm_particles_localdensity(nx, dx, rodo, re0)

    def catalogue(self, capacity):
        """A zeroed page-locked catalogue from a ring of three owned by the
        backend: the one returned by a run stays valid through the next run
        (page-locking fresh memory every run would cost more than the run's
        catalogue copies).  The one after it is zeroed by a helper thread
        while this run goes on: it was returned two runs ago, so its
        validity has ended (numpy's fill releases the GIL)."""
        import threading
        ring = getattr(self, "_cat_ring", None)
        if ring is None or ring[0].capacity != capacity:
            self._cat_join()
            ring = self._cat_ring = [abi.Catalogue(capacity, pinned=True) for _ in range(3)]
            self._cat_next = 0
        self._cat_join()  # this run's catalogue was being zeroed
        c = ring[self._cat_next]
        self._cat_next = (self._cat_next + 1) % 3
        c.reset()  # a no-op when the helper zeroed it
        self._cat_thread = threading.Thread(target=ring[self._cat_next].reset, daemon=True)
        self._cat_thread.start()
        return c

    def _cat_join(self):
        t = getattr(self, "_cat_thread", None)
        if t is not None:
            t.join()
            self._cat_thread = None

    def density(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree=2, fp64=True):
        u1 = np.zeros(nx ** 3, np.float32)
        u11 = np.zeros((max(mesh.total, 1), abi.NAMRX ** 3), np.float32)
        self.a.density(nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, u1, u11)
        return u1.reshape(nx, nx, nx), u11[: mesh.total]

    def renorm_density(self, nx, mesh, fdm, u1, u11):
        u1 = np.ascontiguousarray(u1, np.float32).copy()
        u11 = np.ascontiguousarray(u11, np.float32).copy()
        if u11.shape[0] == 0:
            u11 = np.zeros((1, abi.NAMRX ** 3), np.float32)
        self.a.renorm_density(nx, mesh, fdm, u1, u11)
        return u1, u11[: mesh.total]

    def density_renorm(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, fdm):
        """DENSITY then RENORM_DENSITY with the grids kept on the device
        between the two calls and copied once into page-locked host arrays
        owned by the backend (valid until its next density_renorm).  The copy
        runs on a stream of its own while the caller goes on with the halo
        finder: the arrays hold the grids once sync_outputs() has returned
        (driver.execute calls it before it returns)."""
        import torch
        n11 = max(mesh.total, 1) * abi.NAMRX ** 3
        dev = f"cuda:{self.a.device}"
        self.sync_outputs()  # the previous copy reads the device grids rewritten below
        if getattr(self, "_g1", None) is None or self._g1.numel() != nx ** 3:
            self._g1 = torch.empty(nx ** 3, dtype=torch.float32, device=dev)
            self._h1 = torch.empty(nx ** 3, dtype=torch.float32).pin_memory()
        if getattr(self, "_g11", None) is None or self._g11.numel() < n11:
            self._g11 = torch.empty(n11, dtype=torch.float32, device=dev)
            self._h11 = torch.empty(n11, dtype=torch.float32).pin_memory()
        # both calls return with their work complete on the device
        self.a.density(nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, self._g1, self._g11)
        self.a.renorm_density(nx, mesh, fdm, self._g1, self._g11)
        self._grids_pending = n11
        self._issue_grid_copy()
        u1 = self._h1.numpy().reshape(nx, nx, nx)
        u11 = self._h11[:n11].numpy().reshape(-1, abi.NAMRX ** 3)[: mesh.total]
        return u1, u11

    def _issue_grid_copy(self):
        # on a copy engine, chunk by chunk (the halo finder's short copies on
        # the context stream wait for one chunk at most), after the deferred
        # patch deposit; no SM time is taken from the halo finder
        n11 = getattr(self, "_grids_pending", None)
        if n11 is None:
            return
        self._grids_pending = None
        self.a.copy_to_host_async(self._h1, self._g1)
        self.a.copy_to_host_async(self._h11[:n11], self._g11[:n11])
        self._grids_copying = True

    def sort_x(self, nx, lado0):
        return self.a.sort_dm_particles_x(nx, lado0)

    def sync_outputs(self):
        """Waits for the host copies of the grids left in flight by
        density_renorm."""
        self._issue_grid_copy()
        if getattr(self, "_grids_copying", False):
            self.a.copy_wait()
            self._grids_copying = False

    def tsc_deposit(self, nx, lado0, dx, radx, rote, rete, mesh, fp64=True):
        u1 = np.zeros(nx ** 3, np.float32)
        u11 = np.zeros((max(mesh.total, 1), abi.NAMRX ** 3), np.float32)
        self.a.interpolate_density_tsc(nx, lado0, dx, radx, rote, rete, mesh, u1, u11)
        return u1.reshape(nx, nx, nx), u11[: mesh.total]

    def prune_poor_haloes(self, consts, cat, low1, low2, facrad, do_need_to_count):
        self.a.prune_poor_haloes(consts, cat, low1, low2, facrad, do_need_to_count)

    def halofind_grid_base(self, nx, dx, u1, radx, contrastec, rote, rete, rodo, re0, bound, vol_solap_low, cat,
                           mesh=None, u11=None):
        """HALOFIND_GRID at the base level (haloes_grids.f:287-582); the
        recentering on AMR levels is not on the device (a mesh with patches
        raises)."""
        if mesh is not None and int(np.asarray(mesh.npatch)[1:mesh.nl + 1].sum()) > 0:
            raise AsohfError(8, "HALOFIND_GRID with AMR recentering")
        return self.a.halofind_grid_base(nx, dx, u1, radx, contrastec, rote, rete, rodo, re0, bound, vol_solap_low,
                                         cat)

    def halofind_particles(self, consts, mesh, cat, low1, low2, pph):
        self.a.halofind_particles(consts, mesh, cat, low1, low2)

    def check_rubish(self, cat, low1, low2):
        return self.a.check_rubish(cat, low1, low2)

    def accidental_substructure(self, cat):
        return self.a.accidental_substructure(cat)

    def re_sort_haloes(self, cat, nhallev, ir):
        return self.a.re_sort_haloes(cat, nhallev, ir)

    def overlapping(self, cat, ir, nhallev, vol_solap_low):
        return self.a.overlapping(cat, ir, nhallev, vol_solap_low)

    def substructure_particles(self, consts, mesh, cat, ir, subs_lev, pph):
        self.a.substructure_particles(consts, mesh, cat, ir, subs_lev)

    def final_ids(self, pph, n):
        """PARTICLES_PER_HALO(1:n), fetched once at the end into page-locked
        host memory owned by the backend (valid until its next final_ids)."""
        import torch
        cnt = C.c_int64()
        _check(self.L_len(cnt), "PARTICLES_PER_HALO")
        if self._ids is None or self._ids.shape[0] < max(cnt.value, 1):
            self._ids_t = torch.empty(max(cnt.value, 1), dtype=torch.int32).pin_memory()
            self._ids = self._ids_t.numpy()
        return self.a.particles_per_halo(self._ids)[:n]

    def L_len(self, cnt):
        return self.a.L.asohf_get_particles_per_halo(self.a.h, None, C.c_int64(0), C.byref(cnt), C.c_int(0))

    def poisson_fft(self, u1, dx):
        nx = u1.shape[0]
        u1 = np.ascontiguousarray(u1, np.float32)
        pot = np.zeros_like(u1)
        self.a.poisson_fft(nx, dx, u1, pot)
        return pot


class DeviceBackend(GpuBackend):
    """Backend whose particle input and density grids stay on the GPU
    (torch tensors): nothing crosses PCIe but the catalogue."""

    name = "gpu-device"

    def __init__(self, device: int = 0):
        super().__init__(device)
        self._u1 = None
        self._u11 = None

    def download(self):
        return None

    def sync_outputs(self):
        """The caller's current stream waits for the deferred patch deposit
        (U11 is complete for work issued on it afterwards)."""
        import torch
        self.a.density_wait(torch.cuda.current_stream(self.a.device).cuda_stream)

    def final_ids(self, pph, n):
        """PARTICLES_PER_HALO(1:n), left on the device (a torch tensor owned
        by the backend, valid until its next final_ids)."""
        import torch
        cnt = C.c_int64()
        _check(self.L_len(cnt), "PARTICLES_PER_HALO")
        if self._ids is None or self._ids.shape[0] < max(cnt.value, 1):
            self._ids = torch.empty(max(cnt.value, 1), dtype=torch.int32, device=f"cuda:{self.a.device}")
        return self.a.particles_per_halo(self._ids)[:n]

    def _grids(self, nx, mesh):
        import torch
        n11 = max(mesh.total, 1) * abi.NAMRX ** 3
        if self._u1 is None or self._u1.numel() != nx ** 3:
            self._u1 = torch.empty(nx ** 3, dtype=torch.float32, device=f"cuda:{self.a.device}")
        if self._u11 is None or self._u11.numel() < n11:
            self._u11 = torch.empty(n11, dtype=torch.float32, device=f"cuda:{self.a.device}")
        return self._u1, self._u11

    def density(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree=2, fp64=True):
        u1, u11 = self._grids(nx, mesh)
        self.a.density(nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, u1, u11)
        return u1, u11

    def renorm_density(self, nx, mesh, fdm, u1, u11):
        self.a.renorm_density(nx, mesh, fdm, u1, u11)
        return u1, u11

    def density_renorm(self, nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree, fdm):
        u1, u11 = self.density(nx, lado0, dx, rote, rete, npart_esp, mesh, interp_degree)
        return self.renorm_density(nx, mesh, fdm, u1, u11)
