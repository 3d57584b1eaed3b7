"""CPU checks of two exactness claims the mixed-precision kernels rely on.

1. Ozaki slicing (csrc/panel_scales.cuh, oz_emit_slices): the seven signed
   7-bit slices are taken from the double's exponent and significand with
   integer operations, as sign(v) * (floor(|v| 2^(7p)) mod 2^7).  They must equal
   the slices of the exact FP64 recurrence a_p = trunc(2^7 v), v <- 2^7 v - a_p
   for every |v| < 1, including zeros, subnormals and values next to 1.
2. Refinement residual (csrc/mixed.cu, matern_residual_partial_kernel): the
   lower triangle of 256-row blocks is covered by square super-blocks; every
   pair i > j is applied once to row i and once to column j, every diagonal
   pair once, so the row and column partials add up to C v.  The cover is
   emulated here with small block sizes.
"""
import math

import numpy as np


def _slices_iterative(v):
    out = np.zeros((7, v.size), dtype=np.int64)
    x = v.copy()
    for p in range(7):
        y = x * 128.0
        a = np.trunc(y)
        x = y - a
        out[p] = a.astype(np.int64)
    return out


def _slices_from_bits(v):
    b = v.view(np.int64)
    ex = (b >> 52) & 0x7FF
    sig = (b & ((1 << 52) - 1)) | (1 << 52)
    sh = 1026 - ex
    ok = (ex != 0) & (ex <= 1022) & (sh <= 52)
    mag = np.where(ok, sig >> np.clip(sh, 0, 63), 0)
    neg = b < 0
    out = np.zeros((7, v.size), dtype=np.int64)
    for p in range(1, 8):
        s = (mag >> (49 - 7 * p)) & 127
        out[p - 1] = np.where(neg, -s, s)
    return out


def test_integer_slices_equal_the_fp64_recurrence():
    rng = np.random.default_rng(7)
    n = 200_000
    v = rng.uniform(-1.0, 1.0, n) * np.exp2(rng.integers(-70, 1, n).astype(np.float64))
    edge = np.array([0.0, -0.0, 5e-324, -5e-324, 2.0 ** -1022, np.nextafter(1.0, 0.0), -np.nextafter(1.0, 0.0),
                     2.0 ** -49, -(2.0 ** -49), 2.0 ** -50, 3 * 2.0 ** -50, 0.5, -0.5, 127.0 / 128.0])
    v = np.concatenate([v, edge])
    v = v[np.abs(v) < 1.0]
    assert np.array_equal(_slices_iterative(v), _slices_from_bits(v))


def test_slices_reconstruct_to_2_pow_minus_49():
    rng = np.random.default_rng(8)
    v = rng.uniform(-1.0, 1.0, 10_000)
    s = _slices_from_bits(v).astype(np.float64)
    rec = sum(s[p] * 2.0 ** (-7 * (p + 1)) for p in range(7))
    assert np.max(np.abs(rec - v)) < 2.0 ** -49


def _residual_cover(n, blk, side, c, v):
    nb = (n + blk - 1) // blk
    ns = (nb + side - 1) // side
    rowpart = np.zeros((ns, n))
    colpart = np.zeros((ns, n))
    for lin in range(ns * (ns + 1) // 2):
        sbi = int((math.sqrt(8 * lin + 1) - 1) * 0.5)
        while (sbi + 1) * (sbi + 2) // 2 <= lin:
            sbi += 1
        while sbi * (sbi + 1) // 2 > lin:
            sbi -= 1
        sbj = lin - sbi * (sbi + 1) // 2
        bj0, bj1 = sbj * side, min(nb, sbj * side + side)
        bi0, bi1 = sbi * side, min(nb, sbi * side + side)
        colacc = np.zeros((side, blk))
        for bi in range(bi0, bi1):
            racc = np.zeros(blk)
            for q in range(side):
                bj = bj0 + q
                if bj >= bj1 or bj > bi:
                    break
                jb = bj * blk
                diag = bj == bi
                m = min(blk, n - jb)
                for t in range(blk):
                    i = bi * blk + t
                    if i >= n:
                        continue
                    for jj in range(m):
                        if (not diag) or jj <= t:
                            cij = c[i, jb + jj]
                            racc[t] += cij * v[jb + jj]
                            if (not diag) or jj < t:
                                colacc[q, jj] += cij * v[i]
            for t in range(blk):
                i = bi * blk + t
                if i < n:
                    rowpart[sbj, i] = racc[t]
        for q in range(side):
            for t in range(blk):
                j = (bj0 + q) * blk + t
                if bj0 + q < bj1 and j < n:
                    colpart[sbi, j] = colacc[q, t]
    r = np.zeros(n)
    for i in range(n):
        sb = (i // blk) // side
        r[i] = rowpart[: sb + 1, i].sum() + colpart[sb:ns, i].sum()
    return r


def test_residual_super_blocks_apply_every_pair_once():
    rng = np.random.default_rng(9)
    for n, blk, side in [(37, 4, 2), (64, 8, 3), (5, 4, 2), (100, 7, 4), (33, 8, 1)]:
        a = rng.standard_normal((n, n))
        c = a + a.T
        v = rng.standard_normal(n)
        r = _residual_cover(n, blk, side, c, v)
        assert np.max(np.abs(r - c @ v)) < 1e-12 * max(1.0, np.max(np.abs(c @ v)))
