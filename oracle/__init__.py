"""CPU oracle for the dynamic label-propagation hot path. TEST INFRASTRUCTURE ONLY.

`oracle.ref_np` restates, in NumPy/SciPy, the reference algorithms the CUDA path replaces, each
function citing the reference file:line it follows. It is pinned against golden vectors that were
produced by running the reference itself on the CPU (tests/golden/make_golden.py, committed
fixtures tests/golden/*.npz), and it is used only by tests/, `__graft_entry__.smoke()` and the
CPU-baseline legs of bench.py. Nothing in the product package imports it.
"""
