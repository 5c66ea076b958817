"""Connected components: bit-exact labels against the reference's outputs and the oracle (GPU)."""
import numpy as np
import pytest
import torch

from conftest import golden_csr, load_golden
from dynlplus_b200 import cc
from dynlplus_b200.backend import CSR
from oracle import ref_np as O

pytestmark = pytest.mark.gpu


def T(x):
    return torch.as_tensor(np.ascontiguousarray(x)).cuda()


def test_matches_reference_golden():
    g = load_golden("cc.npz")
    for i in range(int(g["ncases"])):
        n = int(g[f"c{i}_n"])
        lab, nc = cc.connected_components(n, T(g[f"c{i}_rows"]), T(g[f"c{i}_cols"]))
        np.testing.assert_array_equal(lab.cpu().numpy(), g[f"c{i}_labels"])
        assert nc == int(g[f"c{i}_ncomp"])


@pytest.mark.parametrize("n,m", [(1, 0), (10, 5), (100_000, 50_000), (1_000_000, 5_000_000), (2_000_000, 800_000)])
def test_random_graphs_match_oracle(n, m):
    rs = np.random.RandomState(n % 97)
    r, c = rs.randint(0, n, m), rs.randint(0, n, m)
    lab, nc = cc.connected_components(n, T(r.astype(np.int32)), T(c.astype(np.int32)))
    want, wnc = O.connected_components_fast(n, r, c)
    np.testing.assert_array_equal(lab.cpu().numpy(), want)
    assert nc == wnc
    roots = cc.min_vertex_roots(n, T(r.astype(np.int32)), T(c.astype(np.int32)))
    np.testing.assert_array_equal(roots.cpu().numpy(), O.min_vertex_roots(want))


def test_endpoint_out_of_range_is_an_error():
    with pytest.raises(ValueError):
        cc.connected_components(4, T(np.array([0, 7], np.int32)), T(np.array([1, 2], np.int32)))


def test_graph_components_with_sink_match_grounding():
    """The grounding check of Stream._build (dynlp/stream.py:150-159) on the reference's system
    fixture: vertices whose component reaches a labelled vertex are exactly U."""
    g = load_golden("system.npz")
    for b in (0, 2):
        p = f"b{b}"
        A = golden_csr(g, f"{p}_A")
        act, lab = g[f"{p}_active"], g[f"{p}_labeled"]
        G = CSR.from_scipy(A)
        vmask = T((act & ~lab).astype(np.uint8))
        sink = T((act & lab).astype(np.uint8))
        parent, err = cc.graph_components(G, vmask, sink)
        assert int(err.item()) == 0
        par = parent.cpu().numpy()
        n = A.shape[0]
        U = np.flatnonzero((act & ~lab) & (par[:n] == par[n]))
        np.testing.assert_array_equal(U, g[f"{p}_U"])
        assert par[n] == par[par[n]]  # compressed
