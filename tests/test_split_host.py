"""Host checks of the BF16 operand splits behind the tensor-core stages (numpy restatement in
oracle/precision_ref.py; no GPU).

The mixed stage on the tensor cores splits every operand into three BF16 parts and keeps the six products
a_p b_q with p + q <= 2; a two-part split (three products) is kept for comparison.  Stated bounds, on
order-4 reference matrices and random operands of both signs:
  * a three-part split reconstructs an FP32 value to 2^-24 of its magnitude (each part is the BF16 rounding of
    an exact FP32 remainder; the last remainder is at most half a BF16 ulp of the second);
  * six-product matrix products agree with the FP64 product of the same FP32 operands to 2e-7 (relative to
    the sum of absolute terms; measured 1.5e-8 for Dr, 7.6e-9 for LIFT), FP32-level;
  * three-product (two-part) products only to ~2^-16 (measured 1.2e-5, 4.5e-6) — the reason the mixed stage
    uses three parts;
  * the three-part right-hand side of one stage agrees with the FP64 oracle right-hand side to 1e-6 (measured
    1.6e-7, from the FP32 rounding of the operands; two parts: 4.4e-6).
"""
import numpy as np

from oracle import burgers_ref as b
from oracle import oracle as O
from oracle import precision_ref as PR


def _D4():
    ref = b.Problem(4, 3, 1, "sine")
    return ref, ref.el


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0078125, 1e-30, 6.5e4], np.float32)
    h = PR.bf16(x)
    assert np.all(h.view(np.uint32) & 0xFFFF == 0)
    assert np.all(np.abs(x - h) <= 2.0 ** -8 * np.abs(x))
    assert PR.bf16(np.float32(1.00390625)) == np.float32(1.0)  # tie to even
    assert PR.bf16(np.float32(1.005859375)) == np.float32(1.0078125)  # tie to even (odd below)


def test_three_part_split_reconstructs_fp32():
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(100000) * 10.0 ** rng.uniform(-4, 4, 100000)).astype(np.float32)
    p0, p1, p2 = PR.split3(x)
    err = np.abs(x.astype(np.float64) - (p0 + p1 + p2))
    assert np.all(err <= 2.0 ** -24 * np.abs(x.astype(np.float64)))


def test_six_products_carry_fp32_rounding_three_do_not():
    ref, el = _D4()
    rng = np.random.default_rng(11)
    X = rng.standard_normal((256, el.Np)).astype(np.float32)
    F = rng.standard_normal((256, 4 * el.Nfp)).astype(np.float32)
    for M, A in ((el.Dr, X), (el.Ds, X), (el.LIFT, F)):
        exact = A.astype(np.float64) @ np.asarray(M, np.float64).astype(np.float32).astype(np.float64).T
        scale = np.abs(A.astype(np.float64)) @ np.abs(np.asarray(M, np.float64)).T
        e6 = np.max(np.abs(PR.prod6(M, A) - exact) / scale)
        e3 = np.max(np.abs(PR.prod3(M, A) - exact) / scale)
        assert e6 < 2e-7, e6
        assert e3 > 1e-6, e3  # the two-part split is far coarser


def test_three_part_rhs_matches_fp64_rhs():
    ref, el = _D4()
    rng = np.random.default_rng(3)
    u = (0.5 + 0.1 * rng.standard_normal(ref.u0.shape)).reshape(-1)
    hi = u.astype(np.float32)
    lo = (u - hi.astype(np.float64)).astype(np.float32)
    exact = O.RunState(ref).rhs(hi.astype(np.float64) + lo.astype(np.float64))
    got = PR.rhs(ref, hi, lo, parts=3).astype(np.float64).reshape(-1)
    err = np.linalg.norm(got - exact) / np.linalg.norm(exact)
    assert err < 1e-6, err


def test_exact_digit_products_reach_47_bits():
    """The integer-digit products of the precision form (six digits per operand, exact digit sums): the digits
    keep every operand row to 2^-48 of its largest entry (one rounding to nearest) and the dropped digit
    products p + q >= 6 stay below 7 * 2^-46, so against the FP64 product of order-7 reference matrices and
    operands of both signs and varied scales the error is below 2^-42 K max|a_row| max|b_row|."""
    ref = b.Problem(7, 2, 1, "smooth")
    el = ref.el
    rng = np.random.default_rng(3)
    X = rng.standard_normal((40, el.Np)) * np.exp(rng.uniform(-8, 2, (40, 1)))
    for M in (el.Dr, el.LIFT[:, :el.Np]):
        want = X @ M.T
        got = PR.exact_prod(M, X, 6)
        scale = M.shape[1] * np.abs(X).max(axis=1)[:, None] * np.abs(M).max(axis=1)[None, :]
        assert np.max(np.abs(got - want) / scale) < 2.0 ** -42


def test_digits_in_range_for_tiny_entries():
    """Digits stay in their 8-bit ranges (s8 first, u8 after) when a row mixes O(1) values with tiny ones of
    either sign (a floating-point remainder loop would round -1e-18 + 1 to 1 and produce the digit 256), and
    they reconstruct every value to half a unit of the last digit."""
    X = np.array([[1.0, -1.4e-18, 2.5e-17, -0.999999999999, 0.5, -3e-300, 0.0]])
    for S in (4, 6, 7):
        E, d = PR.digits(X, S)
        assert d[0].min() >= -128 and d[0].max() <= 127
        assert all(x.min() >= 0 and x.max() <= 255 for x in d[1:])
        B = 7 + 8 * (S - 1)
        rec = sum(d[p].astype(np.float64) * 2.0 ** (-7 - 8 * p) for p in range(S)) * 2.0 ** E[:, None]
        assert np.max(np.abs(rec - X)) <= 2.0 ** (E.max() - B - 1)
