"""CPU check of the MMA issue schedule of k_conv3 (csrc/conv3x3.cu) for N <= 64, where the three
vertical taps share one MMA: staged row sr feeds accumulator rows lo .. hi = max(sr - 2, rlo) ..
min(sr, rhi) through the stacked B blocks dy = 2, 1, 0 (offset (lo - sr + 2) N rows), and the first
write of accumulator row sr (tap dy = 0, dx = 0, first chunk pair, group 0) is split off without
accumulation. The same index arithmetic, restated here on small random matrices, must give the
direct 3x3 convolution for every row split the kernel uses (one issuer over all R rows, or two
issuers each owning half of them), every chunk-pair count and several input-channel groups, and
no accumulator row may be written by two issuers or read before its first write."""
import numpy as np
import pytest


def schedule(R, N, pairs, groups, issuers, X, Wt):
    """Runs the kernel's MMA sequence; X[g, sr, dx, j] (M x K) staged operands, Wt[g, tap, j] (N x K)."""
    M = X.shape[-2]
    acc = np.full((M, R * N), np.nan)
    owner = np.full(R, -1)
    count = 0

    def mma(h, d0, a, b, accumulate):
        nonlocal count
        count += 1
        for row in range(d0 // N, (d0 + b.shape[0]) // N):
            assert owner[row] in (-1, h), "two issuers write one accumulator row"
            owner[row] = h
        if accumulate:
            assert np.isfinite(acc[:, d0:d0 + b.shape[0]]).all(), "accumulation before the first write"
            acc[:, d0:d0 + b.shape[0]] += a @ b.T
        else:
            acc[:, d0:d0 + b.shape[0]] = a @ b.T

    rows_each = R // issuers
    for h in range(issuers):
        rlo, rhi = h * rows_each, h * rows_each + rows_each - 1
        for g in range(groups):
            for sr in range(rlo, rhi + 3):
                lo, hi = max(sr - 2, rlo), min(sr, rhi)
                n_rows, boff = hi - lo + 1, (lo - sr + 2) * N
                fresh = g == 0 and hi == sr
                for dx in range(3):
                    for j in range(pairs):
                        B = np.concatenate([Wt[g, 3 * (2 - s) + dx, j] for s in range(3)])  # taps dy = 2, 1, 0
                        a = X[g, sr, dx, j]
                        if dx == 0 and j == 0 and fresh:
                            mma(h, sr * N, a, B[2 * N:3 * N], False)
                            if lo < sr:
                                mma(h, lo * N, a, B[boff:boff + (sr - lo) * N], True)
                        else:
                            mma(h, lo * N, a, B[boff:boff + n_rows * N], True)
    return acc.reshape(M, R, N).transpose(1, 0, 2), count


@pytest.mark.parametrize("R,N,issuers", [(8, 16, 1), (8, 32, 1), (8, 32, 2), (8, 16, 2), (4, 64, 1)])
@pytest.mark.parametrize("pairs", [1, 2])
@pytest.mark.parametrize("groups", [1, 3])
def test_stacked_schedule_equals_direct_convolution(R, N, issuers, pairs, groups):
    rng = np.random.default_rng(R * 1000 + N * 10 + issuers + pairs * 7 + groups)
    M, K = 8, 16
    X = rng.standard_normal((groups, R + 2, 3, pairs, M, K))
    Wt = rng.standard_normal((groups, 9, pairs, N, K))
    ref = np.zeros((R, M, N))
    for g in range(groups):
        for o in range(R):
            for dy in range(3):
                for dx in range(3):
                    for j in range(pairs):
                        ref[o] += X[g, o + dy, dx, j] @ Wt[g, 3 * dy + dx, j].T
    got, count = schedule(R, N, pairs, groups, issuers, X, Wt)
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() < 1e-9
    if R == 8 and pairs == 2 and groups == 1:
        assert count == (67 if issuers == 1 else 78)  # against R x 9 x pairs = 144 unstacked
