"""The device generator reproduces the CPU oracle's inputs bit for bit.

bench.py, the command line and the selector's training data generate their matrices on the device
(lt_fill, lt_scale_rows, lt_scale_cols: counter-based, keyed by seed, stream and index); the CPU
oracle generates the same matrices for the parity checks (oracle_fill, oracle_scale_rows/cols). The two
must agree exactly, for every exponent spread and scaling range the configurations use.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,phi,smax,seed", [(257, 300, 0, 0, 1234), (64, 1000, 8, 0, 7),
                                                     (130, 77, 32, 0, 99), (300, 129, 0, 64, 1234),
                                                     (1, 5000, 64, 5, 3)])
def test_device_generator_matches_oracle(cuda, oracle_mod, rows, cols, phi, smax, seed):
    import libthom_b200 as lt

    torch = cuda
    for stream_id in (1, 2, 3):
        X = torch.empty(rows, cols, dtype=torch.float64, device="cuda")
        lt.fill(X, rows * cols, seed, stream_id, phi)
        want = oracle_mod.fill(rows, cols, stream_id, phi, seed)
        if smax:
            lt.scale_rows(X, rows, cols, seed, 4, smax)
            lt.scale_cols(X, rows, cols, seed, 5, smax)
            oracle_mod.scale_rows(want, seed, 4, smax)
            oracle_mod.scale_cols(want, seed, 5, smax)
        torch.cuda.synchronize()
        lt.device_status()
        got = X.cpu().numpy()
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (stream_id, phi, smax)
