"""The solvers' scratch matrices (host logic, on CPU tensors): one buffer per key whatever the row
count, grown by a quarter at least, handed out as row slices with the buffer's leading dimension and
16-byte row starts for padded ones; padding columns stay zero."""
import torch

from dynlplus_b200 import solvers
from dynlplus_b200.backend import ld


def test_scratch_reuses_one_buffer_across_sizes():
    solvers._SCRATCH.clear()
    a = solvers._scratch("t_R", 1000, 9, torch.float32, "cpu")
    assert a.shape == (1000, 9) and ld(a) == 9 and (a == 0).all()
    b = solvers._scratch("t_R", 700, 9, torch.float32, "cpu")  # smaller: a slice of the same buffer
    assert b.shape == (700, 9) and b.data_ptr() == a.data_ptr()
    c = solvers._scratch("t_R", 1100, 9, torch.float32, "cpu")  # larger: grown by a quarter at least
    assert c.shape == (1100, 9) and next(iter(solvers._SCRATCH.values())).shape[0] == 1250
    for n in (10, 1250, 900, 3, 1249):
        assert solvers._scratch("t_R", n, 9, torch.float32, "cpu").shape == (n, 9)
    assert len(solvers._SCRATCH) == 1
    d = solvers._scratch("t_R", 5000, 9, torch.float32, "cpu")  # far larger: exactly what is asked
    assert next(iter(solvers._SCRATCH.values())).shape[0] == 5000 and d.shape == (5000, 9)
    # other keys: columns, dtype, padding, tag
    solvers._scratch("t_R", 100, 10, torch.float32, "cpu")
    solvers._scratch("t_R", 100, 9, torch.float64, "cpu")
    solvers._scratch("t_R", 100, 9, torch.float32, "cpu", padded=True)
    solvers._scratch("t_P", 100, 9, torch.float32, "cpu")
    assert len(solvers._SCRATCH) == 5
    solvers._SCRATCH.clear()


def test_padded_scratch_keeps_its_leading_dimension_and_zero_padding():
    solvers._SCRATCH.clear()
    for C, dt, ldw in ((9, torch.float32, 12), (5, torch.float32, 8), (9, torch.float64, 10), (3, torch.bfloat16, 8)):
        a = solvers._scratch("t_P", 64, C, dt, "cpu", padded=True)
        a.fill_(1)  # a user writes its columns only
        for n in (40, 64, 200):
            v = solvers._scratch("t_P", n, C, dt, "cpu", padded=True)
            assert v.shape == (n, C) and ld(v) == ldw
            assert v.data_ptr() % 16 == 0 and (v.stride(0) * v.element_size()) % 16 == 0
            base = next(t for k, t in solvers._SCRATCH.items() if k[1] == C and k[2] == dt)
            full = base.as_strided((base.shape[0], ldw), (ldw, 1))
            assert (full[:, C:] == 0).all()  # padding columns never written
    solvers._SCRATCH.clear()
