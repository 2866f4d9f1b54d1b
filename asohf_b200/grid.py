"""Grid and background constants the driver computes before the hot path.

Restates, in numpy float32/float64 with the Fortran's per-statement
precision, MALLA (grids.f:2509-2573) with LADO = LADO0 - LADO0/NX
(asohf.f:323), the cosmological background of the driver
(asohf.f:347-364, 440-441) and BRYAN_NORMAN_98 (haloes_grids.f:2-24).
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def malla(nx: int, lado0: float):
    """RADX(0:NX+1) and DX (COMMON /ESPACIADO/)."""
    lado0 = f32(lado0)
    lado = f32(lado0 - f32(lado0 / f32(nx)))
    a = f32(-lado / f32(2.0))
    b = f32(lado / f32(2.0))
    c = f32(f32(b - a) / f32(nx - 1))
    radx = np.zeros(nx + 2, np.float32)
    radx[1] = a
    for i in range(2, nx + 1):
        radx[i] = f32(radx[1] + f32(f32(i - 1) * c))
    radx[0] = f32(radx[1] - c)
    radx[nx + 1] = f32(radx[nx] + c)
    return radx, f32(radx[2] - radx[1])


def cosmology(hubble_h: float, omega0: float, zeta: float) -> dict:
    """PI, ACHE, RODO, RE0, CGR, ROTE, RETE, UV, UM, CONTRASTEC, OMEGAZ."""
    h = f32(hubble_h)
    om = f32(omega0)
    z = f32(zeta)
    pi = f32(math.acos(-1.0))
    ache = f32(float(h) * 3.66e-3)
    rodo = f32(float(om) * 3.0 * float(f32(ache * ache)))
    re0 = f32(f32(1.0) / f32(10.98))
    cgr = f32(1.0 / (8.0 * float(pi)))
    onez = f32(f32(1.0) + z)
    onez3 = f32(f32(onez * onez) * onez)
    rote = f32(rodo * onez3)
    rete = f32(re0 / onez)
    oml = f32(f32(1.0) - om)
    bas = f32(om * onez3)
    omegaz = f32(bas / f32(bas + oml))
    x = f32(omegaz - f32(1.0))
    contrastec = f32(f32(f32(18.0) * f32(pi * pi)) + f32(f32(82.0) * x))
    contrastec = f32(contrastec - f32(f32(39.0) * f32(x * x)))
    contrastec = f32(contrastec / omegaz)
    return dict(pi=pi, ache=ache, rodo=rodo, re0=re0, cgr=cgr, rote=rote, rete=rete,
                uv=f32(299792.458), um=f32(9.1717e18), contrastec=contrastec, omegaz=omegaz)
