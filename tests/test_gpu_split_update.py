"""The split-FP16 tcgen05 off-band update (egs_split_update) against an FP64
torch reference of C -= P_i P_j^T.

Tolerance: |gpu - ref| <= 2e-5 * (|P_i| |P_j|^T + |C|) element-wise (FP32
accumulation over K = ts products of a 2^-22-accurate split); a one-part FP16
or TF32 product would miss this by more than an order of magnitude.
"""
import numpy as np
import pytest

import exageostatcpp_b200 as egs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

RTOL = 2e-5


def tile_slot(i, j, nt):
    return j * nt - j * (j - 1) // 2 + (i - j)


def run_case(ts, nt, band, k, seed):
    g = torch.Generator().manual_seed(seed)
    panel = torch.randn(nt, ts, ts, dtype=torch.float64, generator=g)  # [t][c][r]: column-major tiles
    # rows of very different magnitudes exercise the per-row scaling
    rowmag = 10.0 ** (torch.rand(nt, 1, ts, generator=g, dtype=torch.float64) * 8 - 4)
    panel *= rowmag
    m = nt - band - 1
    nslots = m * (m + 1) // 2
    off = torch.randn(nslots, ts, ts, dtype=torch.float32, generator=g) * 10
    dp, do = panel.cuda(), off.cuda()
    egs.split_update(ts, nt, band, k, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    got = do.cpu()
    mats = panel.transpose(1, 2)  # [t][r][c]
    ref = off.clone().double()
    bound = off.abs().double()
    touched = set()
    for j in range(k + 1, nt):
        for i in range(j + band + 1, nt):
            s = tile_slot(i - band - 1, j, m)
            touched.add(s)
            P = mats[i] @ mats[j].T                      # C[r][c] of the tile as a row-major matrix
            ref[s] -= P.T                                  # stored column-major: [c][r]
            bound[s] += (mats[i].abs() @ mats[j].abs().T).T
    err = (got.double() - ref).abs()
    assert torch.all(err <= RTOL * bound), float((err / bound).max())
    for s in range(nslots):
        if s not in touched:
            assert torch.equal(got[s], off[s])
    return float((err / bound).max())


@pytest.mark.parametrize("ts,nt,band,k", [(256, 5, 1, 0), (256, 4, 0, -1), (512, 6, 2, 0), (256, 7, 2, 2)])
def test_split_update_matches_fp64(ts, nt, band, k):
    worst = run_case(ts, nt, band, k, seed=ts + nt + band + k)
    assert worst < RTOL


def test_split_update_rejects_bad_sizes():
    with pytest.raises(egs.EgsError):
        egs.split_update(192, 4, 1, 0, 0, 0)


def test_split_update_has_no_accumulation_bias():
    # Same-sign products (as in the Cholesky updates of a positively correlated
    # covariance): the tensor core's FP32 accumulation runs short by ~1 ulp per
    # instruction, 8e-6 relative over K = 1024 when accumulated in one pass.
    # Stage-wise promotion to round-to-nearest FP32 keeps the mean signed error
    # at the level of FP32 rounding.
    ts, nt, band = 1024, 3, 0
    g = torch.Generator().manual_seed(1)
    panel = torch.rand(nt, ts, ts, dtype=torch.float64, generator=g) * 0.5 + 0.5
    m = nt - band - 1
    off = torch.zeros(m * (m + 1) // 2, ts, ts, dtype=torch.float32)
    dp, do = panel.cuda(), off.cuda()
    egs.split_update(ts, nt, band, -1, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    got = do.cpu().double()
    mats = panel.transpose(1, 2)
    ref = -(mats[1] @ mats[0].T).T          # target (1, 0), slot 0
    rel = (got[0] - ref) / ref.abs()
    assert abs(float(rel.mean())) < 5e-7, float(rel.mean())
    assert float(rel.pow(2).mean().sqrt()) < 5e-7
