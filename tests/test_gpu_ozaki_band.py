"""The Ozaki-scheme band update (egs_ozaki_band_update: int8 slices, exact
int32 tensor-core products) against an FP64 torch reference of
C_ij -= L_ik L_jk^T on the band targets.

Tolerance: |gpu - ref| <= 1e-12 * (|L_i| |L_j|^T) element-wise.  Seven 7-bit
slices carry 49 bits of every operand relative to its row maximum, so the
expected error is ~1e-14 of the absolute product sum (an FP32-accurate
product would miss the bound by four orders of magnitude).
"""
import numpy as np
import pytest

import exageostatcpp_b200 as egs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

RTOL = 1e-12


def run_case(ts, nt, band, k, seed):
    g = torch.Generator().manual_seed(seed)
    ntp = nt - k
    W = torch.randn(ntp, ts, ts, dtype=torch.float64, generator=g)   # [t][c][r] column-major tiles
    W *= 10.0 ** (torch.rand(ntp, 1, ts, generator=g, dtype=torch.float64) * 6 - 3)  # row magnitudes
    pool = torch.randn(nt * (band + 1), ts, ts, dtype=torch.float64, generator=g)
    dW, dp = W.cuda(), pool.cuda()
    egs.ozaki_band_update(ts, nt, band, k, dW.data_ptr(), dp.data_ptr())
    torch.cuda.synchronize()
    got = dp.cpu()
    rows = W.transpose(1, 2)  # [t][r][c] = L_{k+t,k}(r, c)
    ref = pool.clone()
    bound = torch.zeros_like(pool)
    touched = set()
    for j in range(k + 1, nt):
        for i in range(j, min(nt - 1, j + band) + 1):
            s = j * (band + 1) + (i - j)
            touched.add(s)
            P = rows[i - k] @ rows[j - k].T                 # (r, c) of the target
            A = rows[i - k].abs() @ rows[j - k].abs().T
            if i == j:  # only the lower triangle of a diagonal target is updated
                P = torch.tril(P)
                A = torch.tril(A)
            ref[s] -= P.T                                    # stored column-major [c][r]
            bound[s] += A.T
    err = (got - ref).abs()
    for s in touched:
        assert torch.all(err[s] <= RTOL * bound[s] + 1e-300), float((err[s] / (bound[s] + 1e-300)).max())
    for s in range(nt * (band + 1)):
        if s not in touched:
            assert torch.equal(got[s], pool[s])
    rel = max(float((err[s] / bound[s].clamp_min(1e-300)).max()) for s in touched)
    return rel


@pytest.mark.parametrize("ts,nt,band,k", [(256, 4, 2, 0), (256, 5, 1, 1), (512, 4, 2, 0), (384, 4, 0, 0)])
def test_ozaki_band_update_matches_fp64(ts, nt, band, k):
    worst = run_case(ts, nt, band, k, seed=ts + nt + band + k)
    assert worst < RTOL


def test_mixed_band_methods_agree():
    from oracle import oracle as O
    n, theta = 3000, (1.0, 0.1, 0.5)
    x, y, z = O.load_data(n, 3, theta)
    out = []
    for method in (egs.EGS_BAND_OZAKI_INT8, egs.EGS_BAND_FP64_DMMA):
        p = egs.Problem(n, 256, egs.EGS_PRECISION_MIXED, 2)
        p.set_band_method(method)
        p.set_locations(x, y)
        p.set_observations(z)
        out.append(p.mle_eval(theta))
        p.close()
    (a, la, da), (b, lb, db) = out
    assert abs(a - b) <= 1e-9 * abs(b)
    assert abs(la - lb) <= 1e-9 * abs(lb)
