"""Host-side layout of a mixed-degree batch (no GPU): offsets and concatenated rows."""
import numpy as np


def test_mix_layout(egg):
    from theeggman_b200.hafnian import _mix_layout

    off, flat = _mix_layout([[3, 1], [], [0, 2, 4, 5], [7]])
    assert off.dtype == np.int64 and flat.dtype == np.int32
    assert off.tolist() == [0, 2, 2, 6, 7]
    assert flat.tolist() == [3, 1, 0, 2, 4, 5, 7]
    off, flat = _mix_layout([[], []])
    assert off.tolist() == [0, 0, 0] and flat.size == 0


def test_gbs_mix_shape(egg):
    from theeggman_b200 import workloads as W

    A, idxs = W.gbs_mix(64, 64, range(8, 33, 2), 4)
    assert A.shape == (64, 64) and np.allclose(A, A.T)
    for r in idxs:
        assert len(r) % 2 == 0 and 8 <= len(r) <= 32 and len(set(r.tolist())) == len(r)
