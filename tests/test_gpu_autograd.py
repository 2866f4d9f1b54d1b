"""Differentiable deposit+Poisson: forward against an FP64 numpy restatement,
the hand-written adjoint against the FP64 analytic gradient, and that
gradient against central finite differences (h = 1e-3 cell)."""
import numpy as np
import pytest

from asohf_b200 import grid

pytestmark = pytest.mark.gpu


def tsc_weights64(xp, r, d):
    """TSC weights and derivatives of grids.f:1194-1213 in FP64."""
    w, dw = [], []
    for k, rr in enumerate(r):
        s = xp - rr
        b = np.abs(s) / d
        if k == 1:
            w.append(0.75 - b * b)
            dw.append(-2.0 * b * np.sign(s) / d)
        else:
            t = 1.5 - b
            w.append(0.5 * t * t)
            dw.append(-t * np.sign(s) / d)
    return np.array(w), np.array(dw)


def forward64(x, y, z, m, nx, L, radx, dx, denbas):
    """(rho, pot) for one particle set, FP64."""
    xl = -L / 2
    rho = np.zeros((nx, nx, nx))
    for p in range(x.shape[0]):
        idx, W = [], []
        for v in (x[p], y[p], z[p]):
            i = int((np.float32(v) - np.float32(xl)) / np.float32(dx)) + 1
            i = min(max(i, 1), nx)
            w, _ = tsc_weights64(float(v), [radx[i - 1], radx[i], radx[i + 1]], float(dx))
            idx.append(i)
            W.append(w)
        for kk in range(3):
            for jj in range(3):
                for ii in range(3):
                    a = (idx[0] - 2 + ii) % nx
                    b = (idx[1] - 2 + jj) % nx
                    c = (idx[2] - 2 + kk) % nx
                    rho[c, b, a] += m[p] * W[0][ii] * W[1][jj] * W[2][kk]
    rho /= denbas
    k = np.arange(nx)
    s2 = np.sin(np.pi * k / nx) ** 2
    den = s2[:, None, None] + s2[None, :, None] + s2[None, None, :]
    den[0, 0, 0] = 1e30
    G = -(dx / 2) ** 2 / den
    pot = np.fft.ifftn(np.fft.fftn(rho) * G).real
    return rho, pot, G


def grad64(x, y, z, m, w, nx, L, radx, dx, denbas, G):
    g = np.fft.ifftn(np.fft.fftn(w) * G).real
    xl = -L / 2
    out = np.zeros((3, x.shape[0]))
    for p in range(x.shape[0]):
        idx, W, D = [], [], []
        for v in (x[p], y[p], z[p]):
            i = int((np.float32(v) - np.float32(xl)) / np.float32(dx)) + 1
            i = min(max(i, 1), nx)
            wv, dv = tsc_weights64(float(v), [radx[i - 1], radx[i], radx[i + 1]], float(dx))
            idx.append(i)
            W.append(wv)
            D.append(dv)
        for kk in range(3):
            for jj in range(3):
                for ii in range(3):
                    gv = g[(idx[2] - 2 + kk) % nx, (idx[1] - 2 + jj) % nx, (idx[0] - 2 + ii) % nx]
                    out[0, p] += D[0][ii] * W[1][jj] * W[2][kk] * gv
                    out[1, p] += W[0][ii] * D[1][jj] * W[2][kk] * gv
                    out[2, p] += W[0][ii] * W[1][jj] * D[2][kk] * gv
    return out * m[None, :] / denbas


@pytest.fixture(scope="module")
def setup(gpu_lib):
    import torch
    from asohf_b200.autograd import DepositPoissonLayer
    nx, L = 16, 20.0
    layer = DepositPoissonLayer(nx, L)
    rng = np.random.default_rng(5)
    B, n = 2, 300
    pos = rng.uniform(-L / 2 + 0.5, L / 2 - 0.5, (3, B, n)).astype(np.float32)
    m = rng.uniform(0.5, 1.5, (B, n)).astype(np.float32) * np.float32(1e-8)
    w = rng.standard_normal((B, nx, nx, nx)).astype(np.float32)
    dev = torch.device("cuda:0")
    t = [torch.tensor(a, device=dev) for a in (pos[0], pos[1], pos[2], m)]
    denbas = float(np.float32(layer.dx) ** 3 * layer.rote * layer.rete ** 3)
    return layer, pos, m, w, t, denbas, nx, L


def test_forward_matches_fp64(setup):
    layer, pos, m, w, t, denbas, nx, L = setup
    rho, pot = layer.forward(*t)
    for b in range(pos.shape[1]):
        r64, p64, _ = forward64(pos[0, b], pos[1, b], pos[2, b], m[b].astype(np.float64), nx, L,
                                layer.radx.astype(np.float64), float(layer.dx), denbas)
        assert np.abs(rho[b].cpu().numpy() - r64).max() <= 2e-6 * np.abs(r64).max()
        assert np.abs(pot[b].cpu().numpy() - p64).max() <= 2e-5 * np.abs(p64).max()


def test_adjoint_matches_fp64_gradient_and_fd(setup):
    import torch
    layer, pos, m, w, t, denbas, nx, L = setup
    xs = [a.clone().requires_grad_(True) for a in t[:3]]
    pot = layer(*xs, t[3])
    loss = (pot * torch.tensor(w, device=pot.device)).sum()
    loss.backward()
    gg = np.stack([a.grad.cpu().numpy() for a in xs])
    radx = layer.radx.astype(np.float64)
    dx = float(layer.dx)
    for b in range(pos.shape[1]):
        _, _, G = forward64(pos[0, b][:1], pos[1, b][:1], pos[2, b][:1], m[b][:1].astype(np.float64), nx, L,
                            radx, dx, denbas)
        ref = grad64(pos[0, b], pos[1, b], pos[2, b], m[b].astype(np.float64), w[b].astype(np.float64), nx, L,
                     radx, dx, denbas, G)
        scale = np.abs(ref).max()
        assert np.abs(gg[:, b] - ref).max() <= 1e-4 * scale
        # central differences of the FP64 forward, h = 1e-3 cell, on 5 particles
        h = 1e-3 * dx
        for p in range(5):
            for a in range(3):
                pp = [pos[0, b].astype(np.float64), pos[1, b].astype(np.float64), pos[2, b].astype(np.float64)]
                up = [q.copy() for q in pp]
                dn = [q.copy() for q in pp]
                up[a][p] += h
                dn[a][p] -= h
                lu = (forward64(*up, m[b].astype(np.float64), nx, L, radx, dx, denbas)[1] * w[b]).sum()
                ld = (forward64(*dn, m[b].astype(np.float64), nx, L, radx, dx, denbas)[1] * w[b]).sum()
                fd = (lu - ld) / (2 * h)
                assert abs(fd - ref[a, p]) <= 2e-3 * scale + 1e-3 * abs(ref[a, p]), (b, p, a, fd, ref[a, p])


# ------------------------------------------------------------------ full size
# The differentiable-layer workload at its real size: the 64^3-particle
# snapshot in 8 copies jittered by N(0, 0.01 cell), deposited on a periodic
# 256^3 grid, L = sum(w * phi) with w a seeded N(0, 1) field.  The FP64
# reference is vectorised over particles (numpy, scipy.fft).

def _axis64(v, xl, dx, radx, nx):
    """Host cells (REAL*4 arithmetic as INTERPOLATE_DENSITY_TSC takes them)
    and the TSC weights and derivatives, FP64, for one coordinate array."""
    i = ((v.astype(np.float32) - np.float32(xl)) / np.float32(dx)).astype(np.int64) + 1
    i = np.clip(i, 1, nx)
    v = v.astype(np.float64)
    W, D = [], []
    for k, off in enumerate((-1, 0, 1)):
        s = v - radx[i + off]
        b = np.abs(s) / dx
        if k == 1:
            W.append(0.75 - b * b)
            D.append(-2.0 * b * np.sign(s) / dx)
        else:
            t = 1.5 - b
            W.append(0.5 * t * t)
            D.append(-t * np.sign(s) / dx)
    return i, np.array(W), np.array(D)


def _cells(ix, jy, kz, nx):
    """Flat (z, y, x) indices of the 27 cells of each particle, [27, n]."""
    out = []
    for kk in range(3):
        for jj in range(3):
            for ii in range(3):
                out.append((((kz - 2 + kk) % nx) * nx + (jy - 2 + jj) % nx) * nx + (ix - 2 + ii) % nx)
    return np.array(out)


def _deposit64(x, y, z, m, nx, L, radx, dx, denbas):
    ix, Wx, _ = _axis64(x, -L / 2, dx, radx, nx)
    jy, Wy, _ = _axis64(y, -L / 2, dx, radx, nx)
    kz, Wz, _ = _axis64(z, -L / 2, dx, radx, nx)
    c = _cells(ix, jy, kz, nx)
    w = np.array([Wx[ii] * Wy[jj] * Wz[kk] for kk in range(3) for jj in range(3) for ii in range(3)])
    rho = np.bincount(c.ravel(), (w * m.astype(np.float64)[None, :]).ravel(), minlength=nx ** 3)
    return rho.reshape(nx, nx, nx) / denbas


def _green_half64(nx, dx):
    k = np.arange(nx)
    s2 = np.sin(np.pi * k / nx) ** 2
    den = s2[:, None, None] + s2[None, :, None] + s2[None, None, : nx // 2 + 1]
    den[0, 0, 0] = 1e30
    return -(dx / 2) ** 2 / den


def _solve64(f, G):
    import os
    import scipy.fft as sf
    wk = os.cpu_count() or 1
    return sf.irfftn(sf.rfftn(f, workers=wk) * G, s=f.shape, workers=wk)


def _grad64(x, y, z, m, g, nx, L, radx, dx, denbas):
    ix, Wx, Dx = _axis64(x, -L / 2, dx, radx, nx)
    jy, Wy, Dy = _axis64(y, -L / 2, dx, radx, nx)
    kz, Wz, Dz = _axis64(z, -L / 2, dx, radx, nx)
    c = _cells(ix, jy, kz, nx)
    gv = g.reshape(-1)[c]
    out = np.zeros((3, x.shape[0]))
    q = 0
    for kk in range(3):
        for jj in range(3):
            for ii in range(3):
                out[0] += Dx[ii] * Wy[jj] * Wz[kk] * gv[q]
                out[1] += Wx[ii] * Dy[jj] * Wz[kk] * gv[q]
                out[2] += Wx[ii] * Wy[jj] * Dz[kk] * gv[q]
                q += 1
    return out * m.astype(np.float64)[None, :] / denbas


def _contrib64(px, py, pz, mp, g, nx, L, radx, dx, denbas):
    """<g, rho_p>: the loss carried by particles at (px, py, pz) (arrays)."""
    ix, Wx, _ = _axis64(px, -L / 2, dx, radx, nx)
    jy, Wy, _ = _axis64(py, -L / 2, dx, radx, nx)
    kz, Wz, _ = _axis64(pz, -L / 2, dx, radx, nx)
    c = _cells(ix, jy, kz, nx)
    gv = g.reshape(-1)[c]
    w = np.array([Wx[ii] * Wy[jj] * Wz[kk] for kk in range(3) for jj in range(3) for ii in range(3)])
    return (gv * w).sum(axis=0) * mp.astype(np.float64) / denbas


def test_full_size_gradient(gpu_lib):
    """8 copies x 262144 particles on 256^3: rho and phi against FP64, the
    adjoint gradient of every particle against the FP64 gradient, and that
    gradient against central finite differences (h = 1e-3 cell) of the FP64
    loss on 1000 seeded particles.  Because G is symmetric, L(x) = <w, G rho(x)>
    = <G w, rho(x)> exactly; the differences are taken on the second form
    (only the moved particle's cloud changes), and on two particles also on
    the first form with a full FFT solve per evaluation."""
    import torch
    from asohf_b200 import synth
    from asohf_b200.autograd import DepositPoissonLayer
    s = synth.generate("cfg1")
    L = float(np.float32(s.cfg.lado0))
    nx, B = 256, 8
    layer = DepositPoissonLayer(nx, L)
    dx = float(layer.dx)
    radx = layer.radx.astype(np.float64)
    denbas = float(np.float32(layer.dx) ** 3 * layer.rote * layer.rete ** 3)
    rng = np.random.default_rng(2026)
    base = np.stack([s.x, s.y, s.z]).astype(np.float64)
    pos = base[:, None, :] + rng.normal(0.0, 0.01 * dx, (3, B, base.shape[1]))
    pos = (np.mod(pos + L / 2, L) - L / 2).astype(np.float32)
    m = np.broadcast_to(s.m, (B, s.m.shape[0])).astype(np.float32).copy()
    w = rng.standard_normal((B, nx, nx, nx)).astype(np.float32)
    dev = torch.device("cuda:0")
    xs = [torch.tensor(pos[a], device=dev).requires_grad_(True) for a in range(3)]
    mt = torch.tensor(m, device=dev)
    wt = torch.tensor(w, device=dev)
    rho_g, _ = layer.forward(xs[0].detach(), xs[1].detach(), xs[2].detach(), mt)
    pot_g = layer(*xs, mt)
    (pot_g * wt).sum().backward()
    grad_g = np.stack([a.grad.cpu().numpy() for a in xs])       # (3, B, n)
    rho_g = rho_g.cpu().numpy()
    pot_g = pot_g.detach().cpu().numpy()
    G = _green_half64(nx, dx)
    n = pos.shape[2]
    fd_idx = rng.choice(n, size=1000 // B, replace=False)
    h = 1e-3 * dx
    for b in range(B):
        r64 = _deposit64(pos[0, b], pos[1, b], pos[2, b], m[b], nx, L, radx, dx, denbas)
        assert np.abs(rho_g[b] - r64).max() <= 1e-5 * np.abs(r64).max(), b
        p64 = _solve64(r64, G)
        assert np.abs(pot_g[b] - p64).max() <= 2e-5 * np.abs(p64).max(), b
        g64 = _solve64(w[b].astype(np.float64), G)
        ref = _grad64(pos[0, b], pos[1, b], pos[2, b], m[b], g64, nx, L, radx, dx, denbas)
        scale = np.abs(ref).max()
        assert np.abs(grad_g[:, b] - ref).max() <= 1e-4 * scale, b
        # central differences of the FP64 loss, 125 particles per copy
        p = [pos[a, b, fd_idx].astype(np.float64) for a in range(3)]
        for a in range(3):
            up = [q.copy() for q in p]
            dn = [q.copy() for q in p]
            up[a] += h
            dn[a] -= h
            fd = (_contrib64(*up, m[b, fd_idx], g64, nx, L, radx, dx, denbas)
                  - _contrib64(*dn, m[b, fd_idx], g64, nx, L, radx, dx, denbas)) / (2 * h)
            err = np.abs(fd - ref[a, fd_idx])
            assert (err <= 2e-3 * scale + 1e-3 * np.abs(ref[a, fd_idx])).all(), (b, a, err.max(), scale)
        if b == 0:
            # the first form, L = <w, G rho(x)>, with a full solve per evaluation
            for q in fd_idx[:2]:
                vals = []
                for sgn in (1.0, -1.0):
                    pp = pos[:, b].astype(np.float64).copy()
                    pp[0, q] += sgn * h
                    r = _deposit64(pp[0], pp[1], pp[2], m[b], nx, L, radx, dx, denbas)
                    vals.append((_solve64(r, G) * w[b]).sum())
                fd = (vals[0] - vals[1]) / (2 * h)
                assert abs(fd - ref[0, q]) <= 2e-3 * scale + 1e-3 * abs(ref[0, q]), (q, fd, ref[0, q])
