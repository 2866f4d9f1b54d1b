"""Differentiable TSC deposit + FFT Poisson solve (torch.autograd.Function).

Forward: the base-grid TSC deposit of INTERPOLATE_DENSITY_TSC
(grids.f:1163-1239, periodic, divided by DX^3 ROTE RETE^3) of each of B
particle sets, then MOMENTO + POFFT3D (poisson.f:98-249).  Backward: the
hand-written adjoint in libasohf_gpu.so -- the Green's multiply is real and
symmetric, so dL/drho = G * dL/dphi, and dL/dx_p is the TSC gather of that
field with the derivative weights of particle p.  The reference has no
counterpart: it never differentiates this stage.
"""
from __future__ import annotations

import numpy as np
import torch

from . import grid
from .api import Asohf


class DepositPoissonLayer:
    """Deposit+Poisson on a periodic NX^3 grid of side lado0 (cMpc)."""

    def __init__(self, nx: int, lado0: float, hubble_h: float = 0.678, omega_m: float = 0.31,
                 zeta: float = 0.0, device: int = 0):
        self.nx = nx
        self.lado0 = np.float32(lado0)
        self.radx, self.dx = grid.malla(nx, self.lado0)
        cos = grid.cosmology(hubble_h, omega_m, zeta)
        self.rote, self.rete = cos["rote"], cos["rete"]
        self.lib = Asohf(device)
        self.device = device

    def _sync_stream(self):
        self.lib.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, x, y, z, m):
        """x, y, z, m: (B, n) float32 CUDA tensors -> (rho, pot), (B, NX, NX, NX)."""
        B = x.shape[0]
        nx = self.nx
        rho = torch.empty((B, nx, nx, nx), dtype=torch.float32, device=x.device)
        pot = torch.empty_like(rho)
        self._sync_stream()
        self.lib.tsc_poisson_forward(nx, self.lado0, self.dx, self.radx, self.rote, self.rete,
                                     x.contiguous(), y.contiguous(), z.contiguous(), m.contiguous(),
                                     rho, pot, B)
        return rho, pot

    def adjoint(self, x, y, z, m, w, need_m: bool = True):
        """w = dL/dpot (B, NX, NX, NX) -> dL/dx, dL/dy, dL/dz, dL/dm (B, n)."""
        B = x.shape[0]
        gx, gy, gz = (torch.empty_like(x) for _ in range(3))
        gm = torch.empty_like(m) if need_m else None
        self._sync_stream()
        self.lib.tsc_poisson_adjoint(self.nx, self.lado0, self.dx, self.radx, self.rote, self.rete,
                                     x.contiguous(), y.contiguous(), z.contiguous(), m.contiguous(),
                                     w.contiguous(), gx, gy, gz, gm, B)
        return gx, gy, gz, gm

    def __call__(self, x, y, z, m):
        return DepositPoisson.apply(x, y, z, m, self)


class DepositPoisson(torch.autograd.Function):
    """pot = Poisson(TSC(x, y, z, m)); backward through the library's adjoint."""

    @staticmethod
    def forward(ctx, x, y, z, m, layer: DepositPoissonLayer):
        _, pot = layer.forward(x, y, z, m)
        ctx.save_for_backward(x, y, z, m)
        ctx.layer = layer
        return pot

    @staticmethod
    def backward(ctx, gpot):
        x, y, z, m = ctx.saved_tensors
        gx, gy, gz, gm = ctx.layer.adjoint(x, y, z, m, gpot, need_m=ctx.needs_input_grad[3])
        return gx, gy, gz, gm, None
