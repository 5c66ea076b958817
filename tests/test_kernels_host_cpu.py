"""Host-side helpers of the kernels module (CPU): the reference's lane-group rule and the gather view
that keeps padded score matrices whole."""
import torch

from dynlplus_b200 import kernels, solvers


def test_auto_group_matches_the_reference_rule():
    # dynlp/kernels.py:365-370: the largest power of two <= the mean degree, clamped to [2, 32]
    cases = {0.0: 2, 1.0: 2, 3.9: 2, 4.0: 4, 7.99: 4, 8.0: 8, 10.0: 8, 16.0: 16, 31.9: 16, 32.0: 32, 1e6: 32}
    for deg, g in cases.items():
        assert kernels.auto_group(deg) == g, deg


def test_gather_view_keeps_padded_views_and_copies_short_storage():
    P = solvers.padded_empty(50, 9, torch.float32, "cpu", 0.0)  # 50 x 9 view of a 50 x 12 buffer
    assert kernels.gather_view(P) is P
    rows = P[:20]  # a row slice: the storage still covers 20 x 12 values
    assert kernels.gather_view(rows) is rows
    # a view whose last row's padding lies beyond its storage is copied (the gathers read it)
    base = torch.zeros(12 * 49 + 9)
    short = base.as_strided((50, 9), (12, 1))
    g = kernels.gather_view(short)
    assert g is not short and g.is_contiguous() and torch.equal(g, short)
    dense = torch.zeros(30, 9)
    assert kernels.gather_view(dense) is dense
