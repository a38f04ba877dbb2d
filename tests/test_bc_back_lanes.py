"""CPU check of the b = 64 BC-back schedule (cuev_b200/csrc/backtransform.cu,
bc_back_pipe64_kernel): each column's (TS + 64)-row window is split between two lanes, the upper
one holding window rows [0, TS + 32) and the lower one rows [32, TS + 64); a reflector's dot
product is the sum of the two lanes' 32-term partial sums; each lane updates all of its rows with
the zero-padded reflector (entry k - j + 32 half for its row k); after a hop each lane emits its
rows [0, 32) and the upper lane takes the lower lane's rows [32, 32 + TS) as the next window's
first rows.  Tiles of TS sweeps run from the last to the first, each applying its hop blocks in
increasing order.  This numpy restatement of the schedule (sequential tiles, all columns at once)
must reproduce the oracle's bc_back (the reference's reverse-order application) on the reflectors
of the oracle's own chase."""
import numpy as np
import pytest

from oracle import cuev_oracle as O


def _two_lane_bc_back(U, M, TS):
    b = 64
    n = U.shape[0]
    X = np.array(M, dtype=np.float64, copy=True)
    nsweeps = n - 2
    ntiles = (nsweeps + TS - 1) // TS
    R = TS + 32          # rows per lane
    WS = TS + b          # zero-padded reflector slot
    for t in range(ntiles - 1, -1, -1):
        s0 = t * TS
        top = s0 + 1
        hmax = (n - 1 - top) // b
        first = t + 1 > ntiles - 1
        top_in = top + TS
        hmax_in = -1 if first else (n - 1 - top_in) // b
        Xin = X.copy()   # rows [top_in, n) as tile t + 1 left them
        up = np.zeros((R, X.shape[1]))
        lo = np.zeros((R, X.shape[1]))
        for i in range(TS):
            if top + i < n:
                up[i] = X[top + i]
        for h in range(hmax + 1):
            base = top + h * b
            if first or h <= hmax_in:
                chunk = np.zeros((b, X.shape[1]))
                for i in range(b):
                    r = top_in + b * h + i
                    if r < n:
                        chunk[i] = Xin[r]
                lo[:TS] = chunk[32 - TS:32]
                up[TS:] = chunk[:32]
                lo[TS:] = chunk[32:]
            else:
                lo[:] = 0.0
                up[TS:] = 0.0
            W = np.zeros((TS, WS))
            for j in range(TS):
                for i in range(b):
                    row = base + j + i
                    if s0 + j < nsweeps and row < n:
                        W[j, j + i] = U[row, s0 + j]
            for j in range(TS - 1, -1, -1):
                wu, wl = W[j, :R], W[j, 32:32 + R]
                f = -2.0 * ((wu[j:j + 32, None] * up[j:j + 32]).sum(0)
                            + (wl[j:j + 32, None] * lo[j:j + 32]).sum(0))
                up += wu[:, None] * f[None, :]
                lo += wl[:, None] * f[None, :]
                # both lanes hold window rows [32, 32 + TS) and must agree on them
                assert np.array_equal(up[32:], lo[:TS])
            for i in range(32):
                if base + i < n:
                    X[base + i] = up[i]
                if base + 32 + i < n:
                    X[base + 32 + i] = lo[i]
            up[:TS] = lo[32:32 + TS]
    return X


@pytest.mark.parametrize("n,TS", [(40, 8), (67, 8), (100, 6), (130, 8)])
def test_two_lane_schedule_matches_oracle(n, TS):
    rng = np.random.default_rng(n)
    G = rng.standard_normal((n, n))
    A = (G + G.T) / 2
    B = O.bc_pack(A, 64)
    _, _, U, _ = O.bc_chase(B, 64)
    M = rng.standard_normal((n, 5))
    got = _two_lane_bc_back(U, M, TS)
    want = O.bc_back(U, M, 64)
    assert np.abs(got - want).max() < 1e-13
