"""CPU reference of the learned warm-start network (test infrastructure only).

The warm-start U-Net has no counterpart in the reference project; its
oracle is this plain PyTorch FP32 restatement on the CPU, used by the tests
to check the native forward pass, loss and parameter gradient (autograd) and
the restriction / prolongation around it.  Nothing in the product imports it.

Layout matches the native network: activations NDHWC, weights [27][out][in]
per layer with tap = (dz * 3 + dy) * 3 + dx, layers in the order
c0..c11 of the native file's diagram.  With ``bf16=True`` every stored
activation (and, through autograd of the casts, every stored gradient) is
rounded to BF16 as the GPU stores it, so the comparison isolates summation
order.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

LAYERS = [(16, 16, True), (16, 16, True), (16, 32, True), (32, 32, True), (32, 64, True), (64, 64, True),
          (64, 64, True), (64, 64, True), (64, 32, True), (32, 16, True), (16, 16, True), (16, 16, False)]


def parameter_count() -> int:
    return sum(27 * ci * co for ci, co, _ in LAYERS)


def split_parameters(flat):
    """Flat parameter vector -> list of [27][out][in] tensors."""
    out, off = [], 0
    for ci, co, _ in LAYERS:
        n = 27 * ci * co
        out.append(flat[off:off + n].reshape(27, co, ci))
        off += n
    return out


def _round(x, bf16):
    return x.to(torch.bfloat16).float() if bf16 else x


def _conv(x, w, relu, bf16):
    """x: [B, C, Z, Y, X]; w: [27, out, in]."""
    co, ci = w.shape[1], w.shape[2]
    wt = w.reshape(3, 3, 3, co, ci).permute(3, 4, 0, 1, 2)
    y = F.conv3d(x, wt, padding=1)
    if relu:
        y = torch.relu(y)
    return _round(y, bf16)


def network_input(rhs, bf16=True):
    """rhs [B, Z, Y, X] -> x0 [B, 16, Z, Y, X]: rhs / rms, ones, zeros."""
    b = rhs.shape[0]
    flat = rhs.reshape(b, -1).double()
    rms = torch.sqrt((flat * flat).mean(dim=1))
    inv = torch.where(rms > 0, 1.0 / rms, torch.zeros_like(rms)).float()
    x = torch.zeros((b, 16) + tuple(rhs.shape[1:]), dtype=torch.float32)
    x[:, 0] = rhs.float() * inv.view(b, 1, 1, 1)
    x[:, 1] = 1.0
    return _round(x, bf16)


def forward(weights, x0, bf16=True):
    """Network output [B, 16, Z, Y, X] for input x0 [B, 16, Z, Y, X]."""
    w = weights
    e0a = _conv(x0, w[0], True, bf16)
    e0b = _conv(e0a, w[1], True, bf16)
    p1 = _round(F.avg_pool3d(e0b, 2), bf16)
    e1a = _conv(p1, w[2], True, bf16)
    e1b = _conv(e1a, w[3], True, bf16)
    p2 = _round(F.avg_pool3d(e1b, 2), bf16)
    e2a = _conv(p2, w[4], True, bf16)
    e2b = _conv(e2a, w[5], True, bf16)
    p3 = _round(F.avg_pool3d(e2b, 2), bf16)
    ma = _conv(p3, w[6], True, bf16)
    mb = _conv(ma, w[7], True, bf16)
    u2 = _round(F.interpolate(mb, scale_factor=2, mode="nearest") + e2b, bf16)
    d2 = _conv(u2, w[8], True, bf16)
    u1 = _round(F.interpolate(d2, scale_factor=2, mode="nearest") + e1b, bf16)
    d1 = _conv(u1, w[9], True, bf16)
    u0 = _round(F.interpolate(d1, scale_factor=2, mode="nearest") + e0b, bf16)
    d0 = _conv(u0, w[10], True, bf16)
    return _conv(d0, w[11], False, bf16)


def apply_operator(u, modes):
    """The 7-point pressure operator without solids on u [B, Z, Y, X]; modes
    of the faces x-, x+, y-, y+, z-, z+ (0 fixed value, 1 zero gradient,
    2 periodic): diag counts in-domain or periodic neighbours plus fixed
    faces; (A u) = diag u - sum of neighbours."""
    diag = torch.zeros_like(u)
    acc = torch.zeros_like(u)
    for d, axis in ((0, 3), (1, 2), (2, 1)):
        periodic = modes[2 * d] == 2 and modes[2 * d + 1] == 2
        n = u.shape[axis]
        for side in (0, 1):
            if periodic:
                acc = acc + torch.roll(u, shifts=-1 if side else 1, dims=axis)
                diag = diag + 1.0
                continue
            idx = torch.arange(n, device=u.device)
            inside = ((idx + 1 < n) if side else (idx - 1 >= 0)).to(u.dtype)
            shape = [1, 1, 1, 1]
            shape[axis] = n
            inside = inside.view(shape)
            nb = torch.roll(u, shifts=-1 if side else 1, dims=axis) * inside
            acc = acc + nb
            diag = diag + inside + ((1.0 - inside) if modes[2 * d + side] == 0 else 0.0)
    return diag * u - acc


def loss_and_gradient(flat_params: np.ndarray, rhs: np.ndarray, pressure: np.ndarray, bf16=True, kind="l2", modes=None):
    """Loss and its gradient (flat, FP32), with the weights rounded to BF16
    as the GPU uses them.  rhs, pressure: [B, Z, Y, X].  kind "l2": mean
    (out_0 - p / rms(p))^2; kind "energy": mean over samples of
    1 - (g.Ap)^2 / ((g.Ag)(p.Ap)) with g = out_0 and A the operator of
    ``modes``."""
    p = torch.from_numpy(np.asarray(flat_params, dtype=np.float32))
    pb = p.to(torch.bfloat16).float() if bf16 else p.clone()
    pb.requires_grad_(True)
    w = split_parameters(pb)
    x0 = network_input(torch.from_numpy(rhs), bf16)
    out = forward(w, x0, bf16)[:, 0]
    t = torch.from_numpy(pressure).double()
    b = t.shape[0]
    if kind == "energy":
        g = out.double()
        at = apply_operator(t, modes)
        ag = apply_operator(g, modes)
        s1 = (g * at).reshape(b, -1).sum(1)
        s2 = (g * ag).reshape(b, -1).sum(1)
        s3 = (t * at).reshape(b, -1).sum(1)
        loss = (1.0 - s1 * s1 / (s2 * s3)).mean()
    else:
        rms = torch.sqrt((t.reshape(b, -1) ** 2).mean(dim=1))
        target = (t / rms.view(b, 1, 1, 1)).float()
        loss = ((out - target) ** 2).mean()
    loss.backward()
    return float(loss.detach()), pb.grad.numpy().copy()


def predict(flat_params: np.ndarray, rhs: np.ndarray, bf16=True) -> np.ndarray:
    p = torch.from_numpy(np.asarray(flat_params, dtype=np.float32))
    w = split_parameters(p.to(torch.bfloat16).float() if bf16 else p)
    with torch.no_grad():
        return forward(w, network_input(torch.from_numpy(rhs), bf16), bf16)[:, 0].numpy()


def restrict(fine: np.ndarray, f: int) -> np.ndarray:
    """Sum of the f^3 children of each coarse cell; fine [Z, Y, X]."""
    z, y, x = fine.shape
    return fine.reshape(z // f, f, y // f, f, x // f, f).sum(axis=(1, 3, 5))


def prolong(coarse: np.ndarray, f: int) -> np.ndarray:
    """Trilinear interpolation from coarse to fine cell centres, clamped."""
    out = coarse.astype(np.float64)
    for axis in range(3):
        n = out.shape[axis]
        u = np.clip((np.arange(n * f) + 0.5) / f - 0.5, 0.0, n - 1)
        i0 = np.minimum(np.floor(u).astype(int), n - 1)
        i1 = np.minimum(i0 + 1, n - 1)
        w = u - i0
        shape = [1, 1, 1]
        shape[axis] = n * f
        w = w.reshape(shape)
        out = np.take(out, i0, axis=axis) * (1 - w) + np.take(out, i1, axis=axis) * w
    return out
