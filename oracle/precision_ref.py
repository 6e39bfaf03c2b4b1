"""numpy restatement of the tensor-core stages' right-hand side (test infrastructure only).

Follows the arithmetic of the tensor-core stages (the precision form, parts = 2, and the mixed stage on the
tensor cores, parts = 3): state u = hi + lo (FP32 pair), derivative operand
dw = w - (linear vertex interpolant of w) rounded to FP32, flux in FP32 from the hi traces, both operands and
the matrices split into BF16 parts, products sum_{p+q<=parts-1} A_p B_q (parts = 2: A_hi B_hi + A_hi B_lo +
A_lo B_hi; parts = 3: the six terms of a three-part split), exact products and FP64 sums in place of the tensor
cores' FP32 accumulation, dd = cr ur + cs us + ct ut + L0, rhs = -u dd + LIFT flux.  It
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


def split3(x):
    """Three BF16 parts of FP32 values, each the BF16 rounding of the remainder (remainders exact in FP32)."""
    x = np.asarray(x, np.float32)
    p0 = bf16(x)
    r1 = x - p0
    p1 = bf16(r1)
    p2 = bf16(r1 - p1)
    return p0.astype(np.float64), p1.astype(np.float64), p2.astype(np.float64)


def prod6(M, X):
    """M [rows, K] times X [n, K]^T with the six products a_p b_q, p + q <= 2, of three-part splits (the
    matrix entries rounded to FP32 first, as the packed operands are); returns [n, rows]."""
    Mp = split3(np.asarray(M, np.float64).astype(np.float32))
    Xp = split3(X)
    return sum(Xp[p] @ Mp[q].T for p in range(3) for q in range(3) if p + q <= 2)


def rhs(prob, hi, lo, conservative=0, parts=2):
    """Right-hand side [K, Np] of the tensor-core stage with `parts`-part BF16 splits for the oracle Problem
    `prob` (packed layout)."""
    prod = prod3 if parts == 2 else prod6
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
    ur, us, ut = (prod(D, dw) for D in (el.Dr, el.Ds, el.Dt))
    dd = (cr[:, None] * ur + cs[:, None] * us + ct[:, None] * ut + L0[:, None].astype(np.float64)).astype(np.float32)
    vol = -dd if conservative else -hi * dd
    fm = el.Fmask.reshape(-1)
    uM = hi[:, fm]
    uP = hi.reshape(-1)[np.asarray(prob.vmapP).reshape(K, -1)]
    gf = (g.Fscale * (g.nx + g.ny + g.nz)).astype(np.float32)
    d = uM - uP
    flux = (np.float32(0.5) * d * (np.float32(0.5) * (uM + uP) * gf - np.maximum(np.abs(uM), np.abs(uP)) * np.abs(gf)))
    lift = prod(el.LIFT, flux.astype(np.float32))
    return (vol.astype(np.float64) + lift).astype(np.float32)
