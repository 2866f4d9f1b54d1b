"""The allocation-free base-grid deposit (asohf_density_base_noalloc).

For callers that cannot allocate device memory while they run (an
application that hands all GPU memory to its own pool up front, or code that
must not trigger the synchronisation of cudaMalloc/cudaFree): the entry point
keeps its scratch in a fixed device array.  This test makes the set-up call
first (n = 0: it loads the array and both kernels on the device, the one
call that may need device memory), then calls the entry point through the C
ABI twice in a row on the same inputs -- the second call must clear what the
first left in the shared array -- and checks both results against the
regular entry point, asohf_density.  Both sum each cell's REAL*4 cloud terms
in float64 and round once, but float64 atomics add in no fixed order, so a
cell can differ by the float64 rounding of a different order, which is far
below one float32 ulp: after the final rounding to float32 the results agree
to within 1 ulp of the cell (rtol 2e-7).  The two compute calls must leave
the device's free memory unchanged (cudaMemGetInfo), since they allocate
nothing.  It runs last so that a failure here leaves every other test
already run.
"""
import ctypes as C

import numpy as np
import pytest

from asohf_b200 import abi, api, grid, synth

pytestmark = pytest.mark.gpu

MAX_SIDE = 128  # ASOHF_NOALLOC_MAX_CELLS = 128^3


def test_noalloc_base_deposit_matches_density(gpu_lib):
    import torch
    s = synth.generate("small")
    cfg = s.cfg
    nx = cfg.nx
    L = np.float32(cfg.lado0)
    radx, dx = grid.malla(nx, L)
    cos = grid.cosmology(cfg.h, cfg.omega_m, cfg.zeta)
    n = s.x.shape[0]
    # regular entry point: base grid only (no patches), all particles as species 0
    a = api.Asohf(0)
    a.upload_particles(s.x, s.y, s.z, s.vx, s.vy, s.vz, s.m, s.id)
    npe = np.zeros(abi.N_ESP, np.int32)
    npe[0] = n
    mesh0 = synth.Mesh(0, np.zeros(1, np.int32), *(np.zeros(0, np.int32) for _ in range(6)),
                       *(np.zeros(0, np.float32) for _ in range(3)), np.zeros(0, np.int32))
    ref = np.zeros(nx ** 3, np.float32)
    a.density(nx, L, dx, cos["rote"], cos["rete"], npe, mesh0, 2, ref, np.zeros(1, np.float32))
    a.close()
    # allocation-free entry point, device pointers; every buffer is made first
    L_ = api.load()
    fn = L_.asohf_density_base_noalloc
    fn.restype = C.c_int
    dev = torch.device("cuda:0")
    x, y, z, m = (torch.tensor(v, device=dev) for v in (s.x, s.y, s.z, s.m))
    outs = [torch.full((nx ** 3,), float("nan"), dtype=torch.float32, device=dev) for _ in range(2)]
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call(u1, npart):
        return fn(C.c_int(nx), C.c_float(L), C.c_float(dx), C.c_float(cos["rote"]), C.c_float(cos["rete"]),
                  C.c_int(2), C.c_int64(npart), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                  C.c_void_p(z.data_ptr()), C.c_void_p(m.data_ptr()), C.c_void_p(u1.data_ptr()),
                  C.c_void_p(stream))

    # set-up call: loads the scratch array and the kernels on this device
    assert call(outs[0], 0) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for k in range(2):
        rc = call(outs[k], n)
        assert rc == 0, (k, rc)
        torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    assert free_after == free_before, (free_before, free_after)
    for k in range(2):
        got = outs[k].cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.allclose(got, ref, rtol=2e-7, atol=0), (k, np.abs(got - ref).max())
    # beyond the fixed scratch: a clear refusal (ASOHF_ERR_CAPACITY)
    big = MAX_SIDE + 1
    rc = fn(C.c_int(big), C.c_float(L), C.c_float(dx), C.c_float(cos["rote"]), C.c_float(cos["rete"]),
            C.c_int(2), C.c_int64(0), None, None, None, None, C.c_void_p(outs[0].data_ptr()),
            C.c_void_p(stream))
    assert rc == 3
