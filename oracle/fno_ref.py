"""FP64 PyTorch (CPU) reference of the FNO surrogate, for gradient checks.

TEST INFRASTRUCTURE: the checker, never the product.  The surrogate has no
counterpart in the reference; this restates the network the device kernels
implement from the same flat parameter vector, and autograd supplies exact
gradients to compare with the hand-written backward kernels.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def layout(C: int, m: int, L: int, P: int):
    J = 2 * m
    modes = J * m
    off = {}
    o = 0

    def take(name, n):
        nonlocal o
        off[name] = (o, n)
        o += n

    take("Wl", C * 3)
    take("bl", C)
    for l in range(L):
        take(f"R_{l}", modes * C * C * 2)
        take(f"W_{l}", C * C)
        take(f"b_{l}", C)
    take("Q1", P * C)
    take("b1", P)
    take("Q2", P)
    take("b2", 1)
    return off, o


def forward(params: np.ndarray, masks: np.ndarray, S: int, C: int = 64, m: int = 16, L: int = 4, P: int = 128,
            requires_grad: bool = False):
    """masks: (B, S, S) -> (images (B, S, S) tensor, parameter tensor, input tensor)."""
    off, n = layout(C, m, L, P)
    assert params.size == n
    p = torch.tensor(params, dtype=torch.float64, requires_grad=requires_grad)
    a = torch.tensor(masks, dtype=torch.float64, requires_grad=requires_grad)

    def g(name, shape):
        o, k = off[name]
        return p[o:o + k].reshape(shape)

    B = a.shape[0]
    J = 2 * m
    ys, xs = torch.meshgrid(torch.arange(S, dtype=torch.float64) / S, torch.arange(S, dtype=torch.float64) / S,
                            indexing="ij")
    inp = torch.stack([a, xs.expand(B, S, S), ys.expand(B, S, S)], dim=-1)  # (B, S, S, 3)
    v = inp @ g("Wl", (C, 3)).T + g("bl", (C,))
    kx = torch.arange(m, dtype=torch.float64)
    kyv = torch.tensor([j if j < m else j - J for j in range(J)], dtype=torch.float64)
    xi = torch.arange(S, dtype=torch.float64)
    Ex = torch.exp(-2j * math.pi * torch.outer(kx, xi) / S)          # (m, S)
    Ey = torch.exp(-2j * math.pi * torch.outer(kyv, xi) / S)         # (J, S)
    w = torch.ones(m, dtype=torch.float64)
    w[1:] = 2.0
    for l in range(L):
        R = g(f"R_{l}", (J, m, C, C, 2))
        Rc = torch.complex(R[..., 0], R[..., 1])
        vc = v.to(torch.complex128)
        X = torch.einsum("bysc,ks,jy->bjkc", vc, Ex, Ey)               # (B, J, m, C)
        Y = torch.einsum("bjki,jkio->bjko", X, Rc)
        spec = torch.einsum("bjko,k,ks,jy->byso", Y, w.to(torch.complex128), Ex.conj(), Ey.conj()).real / (S * S)
        z = spec + v @ g(f"W_{l}", (C, C)).T + g(f"b_{l}", (C,))
        v = torch.nn.functional.gelu(z) if l < L - 1 else z
    h = torch.nn.functional.gelu(v @ g("Q1", (P, C)).T + g("b1", (P,)))
    out = h @ g("Q2", (P,)) + g("b2", (1,))
    return out, p, a
