"""Oracle for the learned smoother (test infrastructure only; nothing in the product path imports
this module): the network, its training loss and the sample extraction restated in torch FP64 on
the CPU, with the CUDA library's rounding points.

The reference has no learned smoother (it smooths with weighted Jacobi,
crates/runtime/src/multigrid.rs:245-306); what is restated here is the library's own definition
of the network and the loss, so that the GPU forward, backward and sample kernels can be checked:

- parameters: W1 [16, 3, 3, 3], b1 [16], W2 [16, 16, 3, 3], b2 [16], W3 [1, 16, 3, 3], b3 [1], flat
  in that order (2913 values); weights are rounded to BF16 when used, biases are not;
- network: a1 = bf16(relu(conv(x, W1) + b1)), a2 = bf16(relu(conv(a1, W2) + b2)),
  c = conv(a2, W3) + b3 (cross-correlation, 3 x 3); the BF16 roundings pass gradients straight
  through, as the GPU backward does;
- loss of a sample: (||tH - H c||^2 + lam ||tE - c||^2) / (nH + lam nE) over the 16 x 16 patch,
  H c = c - P R c with R full weighting onto the even points and P bilinear interpolation.
"""
from __future__ import annotations

import numpy as np
import torch

NP = 2913
T = 16


def _bf16(x: torch.Tensor) -> torch.Tensor:
    """Round to BF16 (nearest even) with a straight-through gradient."""
    r = x.detach().to(torch.float32).to(torch.bfloat16).to(torch.float64)
    return x + (r - x).detach()


def unpack(params):
    p = torch.as_tensor(np.asarray(params, dtype=np.float32).astype(np.float64))
    o = 0

    def take(n, shape):
        nonlocal o
        v = p[o:o + n].reshape(shape)
        o += n
        return v

    W1 = take(16 * 3 * 9, (16, 3, 3, 3))
    b1 = take(16, (16,))
    W2 = take(16 * 16 * 9, (16, 16, 3, 3))
    b2 = take(16, (16,))
    W3 = take(16 * 9, (1, 16, 3, 3))
    b3 = take(1, (1,))
    assert o == NP
    return [W1, b1, W2, b2, W3, b3]


def flatten(tensors) -> np.ndarray:
    return torch.cat([t.reshape(-1) for t in tensors]).detach().numpy()


def network(ps, x: torch.Tensor, padding: int = 0) -> torch.Tensor:
    """The network on x [B, 3, H, W]; padding 1 evaluates it on a whole grid with zeros outside."""
    W1, b1, W2, b2, W3, b3 = ps
    conv = torch.nn.functional.conv2d
    a1 = _bf16(torch.relu(conv(x, _bf16(W1), b1, padding=padding)))
    a2 = _bf16(torch.relu(conv(a1, _bf16(W2), b2, padding=padding)))
    return conv(a2, _bf16(W3), b3, padding=padding)


def _fw(c: torch.Tensor) -> torch.Tensor:
    """Full weighting of c [B, 19, 19] (output region [-1, 17]) at the 9 x 9 even loss points."""
    ctr = c[:, 1:18:2, 1:18:2]
    n, s = c[:, 0:17:2, 1:18:2], c[:, 2:19:2, 1:18:2]
    w, e = c[:, 1:18:2, 0:17:2], c[:, 1:18:2, 2:19:2]
    nw, ne = c[:, 0:17:2, 0:17:2], c[:, 0:17:2, 2:19:2]
    sw, se = c[:, 2:19:2, 0:17:2], c[:, 2:19:2, 2:19:2]
    return (4.0 * ctr + (2.0 * ((n + s) + (w + e)) + ((nw + ne) + (sw + se)))) * 0.0625


def _bilinear(rc: torch.Tensor) -> torch.Tensor:
    """Bilinear interpolation of rc [B, 9, 9] to the 16 x 16 loss points."""
    B = rc.shape[0]
    out = torch.zeros(B, T, T, dtype=rc.dtype)
    out[:, 0::2, 0::2] = rc[:, :8, :8]
    out[:, 1::2, 0::2] = 0.5 * (rc[:, :8, :8] + rc[:, 1:9, :8])
    out[:, 0::2, 1::2] = 0.5 * (rc[:, :8, :8] + rc[:, :8, 1:9])
    out[:, 1::2, 1::2] = 0.25 * ((rc[:, :8, :8] + rc[:, 1:9, :8]) + (rc[:, :8, 1:9] + rc[:, 1:9, 1:9]))
    return out


def h_apply(c: torch.Tensor) -> torch.Tensor:
    """H c on the loss patch from c [B, 19, 19]."""
    return c[:, 1:17, 1:17] - _bilinear(_fw(c))


def loss_and_grad(params, inputs, t_h, t_e, n_h, n_e, lam):
    """Mean sample loss and its gradient (flat, FP64) for inputs [B, 3, 25, 25], targets tH, tE
    [B, 16, 16], norms nH, nE [B] and whole-error weight lam."""
    ps = [t.clone().requires_grad_(True) for t in unpack(params)]
    x = torch.as_tensor(np.asarray(inputs, dtype=np.float64))
    th = torch.as_tensor(np.asarray(t_h, dtype=np.float64))
    te = torch.as_tensor(np.asarray(t_e, dtype=np.float64))
    n = torch.as_tensor(np.asarray(n_h, dtype=np.float64) + lam * np.asarray(n_e, dtype=np.float64))
    c = network(ps, x)[:, 0]
    u = th - h_apply(c)
    w = te - c[:, 1:17, 1:17]
    inv = torch.where(n > 0, 1.0 / n, torch.zeros_like(n))
    loss = (((u * u).sum(dim=(1, 2)) + lam * (w * w).sum(dim=(1, 2))) * inv).mean()
    loss.backward()
    return float(loss.detach()), flatten([p.grad for p in ps])


def cd_diag(vx, vy, nu, dx, dy):
    """Diagonal of the steady upwind operator -nu Lap + v.grad (sigma 0, coeff 1), per point."""
    return nu * 2.0 * (1.0 / dx ** 2 + 1.0 / dy ** 2) + np.abs(vx) / dx + np.abs(vy) / dy


def inputs_of(q, vx, vy, d, s, dx, dy):
    """The network's three input channels over a grid (float32 values before the BF16 rounding)."""
    inv_s = 1.0 / s if s > 0 else 0.0
    c0 = (q * inv_s).astype(np.float32)
    c1 = np.where(d != 0, vx * (1.0 / dx) * (1.0 / np.where(d != 0, d, 1.0)), 0.0).astype(np.float32)
    c2 = np.where(d != 0, vy * (1.0 / dy) * (1.0 / np.where(d != 0, d, 1.0)), 0.0).astype(np.float32)
    return np.stack([c0, c1, c2])


def to_bf16(a: np.ndarray) -> np.ndarray:
    return torch.as_tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).numpy()


def extract(q, e, vx, vy, d, s, omega, dx, dy, y0, x0):
    """One sample (inputs [3, 25, 25] as BF16 values, tH, tE [16, 16], nH, nE) at loss origin
    (y0, x0) of grids q, e, vx, vy, d [rows, cols] (FP64)."""
    inp = to_bf16(inputs_of(q, vx, vy, d, s, dx, dy)[:, y0 - 4:y0 + 21, x0 - 4:x0 + 21])
    inv_s = 1.0 / s if s > 0 else 0.0

    def hh(f):
        c = torch.as_tensor(f[None, y0 - 1:y0 + 18, x0 - 1:x0 + 18].copy())
        return h_apply(c)[0].numpy()

    he, hq = hh(e), hh(q)
    ep, qp = e[y0:y0 + T, x0:x0 + T], q[y0:y0 + T, x0:x0 + T]
    return (inp, (he - omega * hq) * inv_s, (ep - omega * qp) * inv_s, float(np.sum(he * he) * inv_s * inv_s),
            float(np.sum(ep * ep) * inv_s * inv_s))


def smooth_step(params, x, b_minus_ax_over_d, vx, vy, d, omega, dx, dy):
    """One learned step on a whole grid given q = (b - A x) / d (0 on the ring): returns
    (x + omega q + s c on the interior, c, s)."""
    q = b_minus_ax_over_d
    rows, cols = q.shape
    s = float(np.sqrt(np.sum(q[1:-1, 1:-1] ** 2) / ((rows - 2) * (cols - 2))))
    inp = to_bf16(inputs_of(q, vx, vy, d, s, dx, dy)).astype(np.float64)
    with torch.no_grad():
        c = network(unpack(params), torch.as_tensor(inp[None]), padding=1)[0, 0].numpy()
    out = x.copy()
    out[1:-1, 1:-1] = x[1:-1, 1:-1] + omega * q[1:-1, 1:-1] + s * c[1:-1, 1:-1]
    return out, c, s
