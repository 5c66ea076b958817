"""Connected components on the device (dynlp/cc.py:8-23).

`connected_components(n, rows, cols)` returns (int32 labels in [0, n_comp), n_comp) with the
reference's canonical numbering: components ranked by their smallest vertex id (the reference's
`unique(..., return_inverse=True)` relabel, cc.py:22). The kernel is a lock-free union-find
(hook larger root under smaller, path halving) rather than the reference's host-synchronised
hook/jump rounds; the labels are identical bit for bit.
"""
from __future__ import annotations

import torch

from . import _lib
from .backend import code, ptr, stream, workspace


def min_vertex_roots(n, rows, cols) -> torch.Tensor:
    """parent[v] = smallest vertex id in v's component (int32, device)."""
    rows = rows.to(torch.int32).contiguous()
    cols = cols.to(torch.int32).contiguous()
    dev = rows.device
    parent = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call("dlp_cc_edges", int(n), ptr(rows), ptr(cols), int(rows.numel()), ptr(parent), ptr(err), stream())
    if int(err.item()):
        raise ValueError("connected_components: edge endpoint outside [0, n)")
    return parent[:n]


def relabel(parent: torch.Tensor, sync: bool = True):
    """Rank of each root among the roots (unique + inverse); returns (labels, n_comp)."""
    n = int(parent.numel())
    label = torch.empty(max(n, 1), dtype=torch.int32, device=parent.device)
    nc = torch.empty(1, dtype=torch.int32, device=parent.device)
    ws = workspace("compact").get(_lib.lib().dlp_compact_workspace_bytes(n))
    _lib.call("dlp_cc_relabel", n, ptr(parent), ptr(label), ptr(nc), ptr(ws), ws.numel(), stream())
    return (label[:n], int(nc.item())) if sync else (label[:n], nc)


def connected_components(n, rows, cols):
    """(labels in [0, n_comp), n_comp) for an undirected edge list (dynlp/cc.py:8-23)."""
    if n == 0:
        dev = rows.device if torch.is_tensor(rows) else None
        return torch.zeros(0, dtype=torch.int32, device=dev), 0
    return relabel(min_vertex_roots(n, rows, cols))


def graph_components(G, vmask=None, sink=None, w=None):
    """Min-vertex-id roots over the stored entries of a row-range graph with a sink vertex n.

    Entry (u, v) joins u and v when vmask[u] and vmask[v] (and w != 0 when w is given); it joins
    u and the sink when vmask[u] and sink[v]. Returns parent of length n + 1 (device int32).
    This is the grounding check of dynlp/stream.py:150-159 and :275-280 in one launch.
    """
    n = G.shape[0]
    dev = G.indices.device
    parent = torch.empty(n + 1, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = workspace("cc_graph").get(_lib.lib().dlp_cc_graph_workspace_bytes())
    _lib.call("dlp_cc_graph", n, ptr(G.rbeg), ptr(G.rend), ptr(G.indices), ptr(w),
              code(w) if w is not None else 0, ptr(vmask), ptr(sink), ptr(parent), ptr(err), ptr(ws), ws.numel(),
              stream())
    return parent, err


def ground_reach(G, vmask, sink, umask, in_t, w=None):
    """Grounded set of the graph form of graph_components, updated in place: umask[u] = 1 iff
    vmask[u] and u's component reaches the sink (the vertices whose root is the sink's root there);
    in_t[u] = 1 where membership changed. Bottom-up reachability sweeps; the union-find finishes
    the job when they do not settle. Returns (number of changes, sweeps run; negative = fallback)."""
    import ctypes as ct
    n = G.shape[0]
    dev = G.indices.device
    ce = torch.zeros(2, dtype=torch.int32, device=dev)  # [changes, error]: read back together
    cnt, err = ce[0:1], ce[1:2]
    sweeps = ct.c_int32(0)
    ws = workspace("ground_reach").get(_lib.lib().dlp_ground_reach_workspace_bytes(n))
    rbeg, rend = (G.rbeg, G.rend) if hasattr(G, "rbeg") else (G.indptr[:-1], G.indptr[1:])
    _lib.call("dlp_ground_reach", n, ptr(rbeg), ptr(rend), ptr(G.indices), ptr(w), code(w) if w is not None else 0,
              ptr(vmask), ptr(sink), ptr(umask), ptr(in_t), ptr(cnt), ptr(err), ct.addressof(sweeps), ptr(ws),
              ws.numel(), stream())
    changes, bad = ce.tolist()
    if bad:
        raise ValueError("ground_reach: entry column outside [0, n)")
    return changes, int(sweeps.value)



# ---------------------------------------------------------------------------------------------
# adaptive components of new vertices (dynlp/cc.py:26-83)
# ---------------------------------------------------------------------------------------------
def _lightest(nc, cu, cv, de):
    """Per component with an outgoing edge: (component, the other side, weight) of its lightest one,
    ties to the smallest other side (dynlp/cc.py:26-34). min-reductions: order-independent."""
    dev = cu.device
    best = torch.full((nc,), float("inf"), dtype=torch.float32, device=dev)
    best.scatter_reduce_(0, cu, de, "amin")
    nb = torch.full((nc,), nc, dtype=torch.int64, device=dev)
    sel = de <= best[cu]
    nb.scatter_reduce_(0, cu[sel], cv[sel], "amin")
    c = torch.nonzero(nb < nc, as_tuple=False).flatten()
    return c, nb[c], best[c]


def fh_components(m, rows, cols, d, k, ground=None):
    """Felzenszwalb-Huttenlocher merging in Boruvka rounds (dynlp/cc.py:37-73): each round every
    component takes its lightest outgoing edge and merges across it when d(e) <= min over both
    sides of Int(C) + k/|C| (Int = largest internal dissimilarity, fp32 as the reference keeps it);
    with `ground`, components holding none then join their lightest neighbour until every one has
    some. The merges of a round are one call of the component kernel (rank labels)."""
    dev = rows.device
    lab = torch.arange(m, dtype=torch.int64, device=dev)
    Int = torch.zeros(m, dtype=torch.float32, device=dev)
    size = torch.ones(m, dtype=torch.float32, device=dev)
    rows, cols, d = rows.long(), cols.long(), d.to(torch.float32)
    g_v = ground.to(torch.float32) if ground is not None else None
    nc, fh = m, True
    while rows.numel():
        cu, cv = lab[rows], lab[cols]
        ext = cu != cv
        if not fh:
            g = torch.zeros(nc, dtype=torch.float32, device=dev).index_add_(0, lab, g_v)
            ext &= g[cu] == 0
        if not bool(ext.any()):
            break
        c, t, dc = _lightest(nc, cu[ext], cv[ext], d[ext])
        if fh:
            ok = dc <= torch.minimum(Int[c] + k / size[c], Int[t] + k / size[t])
            if not bool(ok.any()):
                if g_v is None:
                    break
                fh = False
                continue
            c, t, dc = c[ok], t[ok], dc[ok]
        root, nc = connected_components(nc, c.to(torch.int32), t.to(torch.int32))
        root = root.long()
        Int2 = torch.zeros(nc, dtype=torch.float32, device=dev).scatter_reduce_(0, root, Int, "amax")
        Int2.scatter_reduce_(0, root[c], dc, "amax")
        size2 = torch.zeros(nc, dtype=torch.float32, device=dev).index_add_(0, root, size)
        lab, Int, size = root[lab], Int2, size2
    return lab.to(torch.int32), nc


def adaptive_components(m, rows, cols, w, s_r, s_c, wmax, ground=None):
    """Component-adaptive merging of the new vertices (dynlp/cc.py:76-83): dissimilarity
    1 - w/wmax scaled by the endpoints' own mean dissimilarities, k = its mean."""
    if m == 0:
        return torch.zeros(0, dtype=torch.int32, device=rows.device), 0
    d = (1 - w / wmax) / torch.sqrt(s_r * s_c)
    k = float(d.double().mean().item()) if d.numel() else 0.0
    return fh_components(m, rows, cols, d, k, ground)
