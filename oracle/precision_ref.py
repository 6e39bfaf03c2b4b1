"""numpy restatement of the precision form's right-hand side (test infrastructure only).

Follows the arithmetic of the tensor-core stage: state u = hi + lo (FP32 pair), derivative operand
dw = w - (linear vertex interpolant of w) rounded to FP32, flux in FP32 from the hi traces, both operands and
the matrices split into BF16 hi/lo, products A_hi B_hi + A_hi B_lo + A_lo B_hi (exact products, FP64 sums in
place of the tensor cores' FP32 accumulation), dd = cr ur + cs us + ct ut + L0, rhs = -u dd + LIFT flux.  It
exists to check the GPU kernel's logic where the split itself is inaccurate (order 7 with the reference's node
set), so a comparison against FP64 alone cannot tell a kernel error from the precision limit.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    return (((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16).astype(np.uint32).view(np.float32)


def split(x):
    x = np.asarray(x, np.float32)
    h = bf16(x)
    return h.astype(np.float64), bf16(x - h).astype(np.float64)


def prod3(M, X):
    """M [rows, K] times X [n, K]^T with the three split products; returns [n, rows]."""
    Mh, Ml = split(M)
    Xh, Xl = split(X)
    return Xh @ Mh.T + Xl @ Mh.T + Xh @ Ml.T


def rhs(prob, hi, lo, conservative=0):
    """Right-hand side [K, Np] of the precision form for the oracle Problem `prob` (packed layout)."""
    el, g = prob.el, prob.geo
    K, Np = prob.K, el.Np
    hi = np.asarray(hi, np.float32).reshape(K, Np)
    lo = np.asarray(lo, np.float32).reshape(K, Np)
    u = hi.astype(np.float64) + lo.astype(np.float64)
    w = 0.5 * u * u if conservative else u
    r, s, t = el.r, el.s, el.t
    vt = [int(np.argmin((r - a) ** 2 + (s - b) ** 2 + (t - c) ** 2))
          for a, b, c in ((-1, -1, -1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
    lam = np.stack(((1 + r) / 2, (1 + s) / 2, (1 + t) / 2), 1)
    wA = w[:, vt[0]]
    dB, dC, dD = (w[:, vt[k]] - wA for k in (1, 2, 3))
    dw = ((w - wA[:, None]) - (lam[None, :, 0] * dB[:, None] + lam[None, :, 1] * dC[:, None]
                              + lam[None, :, 2] * dD[:, None])).astype(np.float32)
    cr = (g.rx + g.ry + g.rz)[:, 0].astype(np.float32).astype(np.float64)
    cs = (g.sx + g.sy + g.sz)[:, 0].astype(np.float32).astype(np.float64)
    ct = (g.tx + g.ty + g.tz)[:, 0].astype(np.float32).astype(np.float64)
    L0 = np.float32(0.5) * (cr * dB + cs * dC + ct * dD).astype(np.float32)
    ur, us, ut = (prod3(D, dw) for D in (el.Dr, el.Ds, el.Dt))
    dd = (cr[:, None] * ur + cs[:, None] * us + ct[:, None] * ut + L0[:, None].astype(np.float64)).astype(np.float32)
    vol = -dd if conservative else -hi * dd
    fm = el.Fmask.reshape(-1)
    uM = hi[:, fm]
    uP = hi.reshape(-1)[np.asarray(prob.vmapP).reshape(K, -1)]
    gf = (g.Fscale * (g.nx + g.ny + g.nz)).astype(np.float32)
    d = uM - uP
    flux = (np.float32(0.5) * d * (np.float32(0.5) * (uM + uP) * gf - np.maximum(np.abs(uM), np.abs(uP)) * np.abs(gf)))
    lift = prod3(el.LIFT, flux.astype(np.float32))
    return (vol.astype(np.float64) + lift).astype(np.float32)
