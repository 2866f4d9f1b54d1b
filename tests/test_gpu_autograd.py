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
