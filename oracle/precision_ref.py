"""numpy restatements of the tensor-core stages' right-hand sides (test infrastructure only).

1. BF16 splits (`rhs`, parts = 2 or 3): the arithmetic of the mixed stage on the tensor cores (orders 1..4,
   three parts): state u = hi + lo (FP32 pair), derivative operand dw = w - (linear vertex interpolant of w)
   rounded to FP32, flux in FP32 from the hi traces, both operands and the matrices split into BF16 parts,
   products sum_{p+q<=parts-1} A_p B_q, exact products and FP64 sums in place of the tensor cores' FP32
   accumulation, dd = cr ur + cs us + ct ut + L0, rhs = -u dd + LIFT flux.  Two parts are kept to show why the
   mixed stage needs three.
2. Exact integer digits (`rhs_exact`, `stage_exact`): the precision form at orders 4..7, whose products are
   exact sums of 8-bit digit products; restated with numpy int64 products, so the GPU kernel can be checked to
   FP64 rounding even where the reference's node set makes every FP32-level product lose the derivative.
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


# ------------------------------------------------------------------------------------------------------------
# Exact integer-digit products (the precision form at orders 4..7): restatement of the tensor-core kernel's
# arithmetic with numpy int64 products.
# ------------------------------------------------------------------------------------------------------------
def digits(X, S):
    """Row exponents E (|x| < 2^E per row; 0 for all-zero rows) and S digits of X [rows, K]: every value rounded
    once to n = rint(x 2^(B-E)), B = 7 + 8 (S - 1) (clamped to 2^B - 1 at the top), then cut by integer shifts,
    x ~ 2^(E-7) (d_0 + 2^-8 (d_1 + ...)), d_0 = n >> (B - 7) in [-128, 127], d_p = byte p of n in [0, 255]."""
    X = np.asarray(X, np.float64)
    B = 7 + 8 * (S - 1)
    m = np.abs(X).max(axis=1)
    E = np.where(m > 0, np.frexp(np.where(m > 0, m, 1.0))[1], 0).astype(np.int64)
    n = np.rint(X * np.ldexp(1.0, B - E)[:, None]).astype(np.int64)
    n = np.minimum(n, (1 << B) - 1)
    ds = [n >> (B - 7)] + [(n >> (8 * (S - 1 - p))) & 0xff for p in range(1, S)]
    return E, ds


def exact_prod(M, X, S):
    """X [n, K] times M [rows, K]^T with S-digit operands: the digit products d^X_q d^M_p with p + q <= S - 1
    summed exactly (int64), levels joined by Horner's rule in FP64 and scaled by 2^(E_X + E_M - 14)."""
    EM, dm = digits(M, S)
    EX, dx = digits(X, S)
    h = np.zeros((X.shape[0], M.shape[0]))
    for L in range(S - 1, -1, -1):
        acc = sum(dx[q] @ dm[L - q].T for q in range(L + 1))
        h = h * 0.00390625 + acc.astype(np.float64)
    return h * np.ldexp(1.0, (EX[:, None] + EM[None, :] - 14))


def rhs_exact(prob, hi, lo, S=6, conservative=0, el=None, geo=None):
    """Right-hand side [K, Np] of the exact-digit precision stage for the oracle Problem `prob`: u = hi + lo
    (FP64), dw and the Lax-Friedrichs flux in FP64, the metric sums and face factors rounded to FP32 (the
    stage's compact geometry), the volume product [cr dw | cs dw | ct dw] x [Dr | Ds | Dt]^T and the LIFT product
    with exact_prod.  `el` (optional) supplies the reference element's nodes r, s, t and matrices Dr, Ds, Dt,
    LIFT in place of the oracle's own: on the reference's node set two FP64 constructions of LIFT agree only to
    ~1e-5 at order 7, so a kernel is checked with the operators it was given; `geo` (optional) likewise supplies
    the per-node metrics rx..tz and face arrays nx, ny, nz, Fscale whose FP32-rounded sums the stage uses."""
    g = prob.geo if geo is None else geo
    el = prob.el if el is None else el
    K, Np = prob.K, el.Np
    u = (np.asarray(hi, np.float32).astype(np.float64) + np.asarray(lo, np.float32).astype(np.float64)).reshape(K, Np)
    w = 0.5 * u * u if conservative else u
    r, s, t = el.r, el.s, el.t
    vt = [int(np.argmin((r - a) ** 2 + (s - b) ** 2 + (t - c) ** 2))
          for a, b, c in ((-1, -1, -1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
    lam = np.stack(((1 + r) / 2, (1 + s) / 2, (1 + t) / 2), 1)
    wA = w[:, vt[0]]
    dB, dC, dD = (w[:, vt[k]] - wA for k in (1, 2, 3))
    dw = (w - wA[:, None]) - (lam[None, :, 0] * dB[:, None] + lam[None, :, 1] * dC[:, None]
                              + lam[None, :, 2] * dD[:, None])
    c = [(getattr(g, a + "x") + getattr(g, a + "y") + getattr(g, a + "z"))[:, 0].astype(np.float32).astype(np.float64)
         for a in ("r", "s", "t")]
    L0 = 0.5 * (c[0] * dB + c[1] * dC + c[2] * dD)
    Bv = np.concatenate([c[d][:, None] * dw for d in range(3)], axis=1)
    dd = exact_prod(np.concatenate((el.Dr, el.Ds, el.Dt), axis=1), Bv, S) + L0[:, None]
    fm = el.Fmask.reshape(-1)
    uM = u[:, fm]
    uP = u.reshape(-1)[np.asarray(prob.vmapP).reshape(K, -1)]
    Nfp = el.Nfp
    gfull = g.Fscale * (g.nx + g.ny + g.nz)
    gf = np.repeat(gfull[:, ::Nfp].astype(np.float32).astype(np.float64), Nfp, axis=1)  # per face, FP32
    d = uM - uP
    flux = 0.5 * d * (0.5 * (uM + uP) * gf - np.maximum(np.abs(uM), np.abs(uP)) * np.abs(gf))
    lift = exact_prod(el.LIFT, flux, S)
    return (-dd if conservative else -u * dd) + lift


def stage_exact(prob, hi, lo, resu, a, b, dt, S=6, conservative=0, el=None, geo=None):
    """One stage of the exact-digit precision form: resu = fp32(a resu + dt rhs), u = u + b resu (FP64), u split
    back into the (hi, lo) FP32 pair.  Returns (hi, lo, resu) flat."""
    rhs = rhs_exact(prob, hi, lo, S, conservative, el, geo).reshape(-1)
    u = np.asarray(hi, np.float32).astype(np.float64) + np.asarray(lo, np.float32).astype(np.float64)
    rn = (a * np.asarray(resu, np.float32).astype(np.float64) + dt * rhs).astype(np.float32)
    un = u + b * rn.astype(np.float64)
    h = un.astype(np.float32)
    return h, (un - h.astype(np.float64)).astype(np.float32), rn
