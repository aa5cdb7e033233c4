"""Split-node connectivity between bones (host preprocessing of the solve inputs).

Same result, bit for bit, as the reference's ``split_connectivity_fast`` (rb/splitfe.py:261-305, itself
equal to ``split_connectivity`` :17-55):

* a grid node touched by bone cells of two or more bones is split, one copy per bone;
* the lowest bone id keeps the grid id; the other (node, bone) pairs get ids nnode, nnode+1, ...
  in ascending (node, bone) order, and ``orig`` maps every id back to its grid node;
* a bone cell uses its own bone's copy; a joint / soft cell (part 0) at a split node uses the copy of
  the bone with the largest share in the cell (first maximum in ascending bone order) when that share
  is positive, otherwise the bone with the most bone cells at the node (first maximum).
"""
import numpy as np


def split_connectivity(g, active, part, bone_share):
    """Returns (cn (ncell, 8) int64, orig (nnew,) int64, number of split grid nodes)."""
    nnode = g.nnode
    nb = bone_share.shape[1]
    act = np.flatnonzero(active)
    part = np.asarray(part)
    corners = g.cell_nodes[act]                                        # (n, 8)
    pc = part[act].astype(np.int64)
    # (node, bone) incidences of bone cells, sorted by node then bone, with their multiplicity
    isb = pc > 0
    inc = (corners[isb] * nb + pc[isb, None]).ravel()
    pair, mult = np.unique(inc, return_counts=True)
    pnode = pair // nb
    pbone = pair - pnode * nb
    per_node = np.bincount(pnode, minlength=nnode)
    split = per_node >= 2
    lead = np.ones(len(pair), bool)
    lead[1:] = pnode[1:] != pnode[:-1]
    extra = split[pnode] & ~lead
    new_id = np.where(extra, nnode + np.cumsum(extra) - 1, -1)
    orig = np.concatenate([np.arange(nnode, dtype=np.int64), pnode[extra]])
    cn = g.cell_nodes.copy()
    rr, ll = np.nonzero(split[corners])
    if len(rr) == 0:
        return cn, orig, int(split.sum())
    node = corners[rr, ll]
    cell = act[rr]
    bone = pc[rr].copy()
    # joint / soft cells: choose among the node's bones (a contiguous run of ``pair`` starting at ``first``)
    soft = np.flatnonzero(bone == 0)
    if len(soft):
        first = np.searchsorted(pnode, node[soft])
        cnt = per_node[node[soft]]
        width = int(cnt.max())
        j = np.arange(width)
        valid = j[None, :] < cnt[:, None]
        idx = np.where(valid, first[:, None] + j[None, :], 0)
        cand = pbone[idx]
        shares = np.where(valid, bone_share[cell[soft][:, None], cand], -np.inf)
        mults = np.where(valid, mult[idx], -1)
        by_share = cand[np.arange(len(soft)), np.argmax(shares, 1)]
        by_count = cand[np.arange(len(soft)), np.argmax(mults, 1)]
        bone[soft] = np.where(shares.max(1) > 0, by_share, by_count)
    nid = new_id[np.searchsorted(pair, node * nb + bone)]
    take = nid >= 0
    cn[cell[take], ll[take]] = nid[take]
    return cn, orig, int(split.sum())


def split_connectivity_device(g, active, part, bone_share):
    """The same connectivity computed on the device (libfeb200 ``feb_split_connectivity``): returns
    (cn (ncell, 8) int64, orig (nnew,) int64, number of split grid nodes), equal bit for bit to
    ``split_connectivity`` and to the reference's."""
    import ctypes as C
    from . import _lib
    from .engine import _dev, _grid_struct, _host, _ptr, _stream, _torch
    torch = _torch()
    share = np.asarray(bone_share, np.float64)
    nb = share.shape[1]
    act = _dev(np.asarray(active, bool).view(np.uint8).ravel(), np.uint8)
    pt = _dev(np.asarray(part).ravel(), np.int32)
    sh = _dev(share.ravel(), np.float64)
    gs = _grid_struct(g)
    lib = _lib.load()
    ntot, nspl = C.c_int64(), C.c_int64()
    _lib.check(lib.feb_split_connectivity(C.byref(gs), _ptr(act), _ptr(pt), _ptr(sh), nb, None, None, 0, C.byref(ntot),
                                          C.byref(nspl), _stream()))
    cn = torch.empty(8 * g.ncell, dtype=torch.int64, device="cuda")
    orig = torch.empty(ntot.value, dtype=torch.int64, device="cuda")
    _lib.check(lib.feb_split_connectivity(C.byref(gs), _ptr(act), _ptr(pt), _ptr(sh), nb, _ptr(cn), _ptr(orig),
                                          ntot.value, C.byref(ntot), C.byref(nspl), _stream()))
    cn_h, orig_h = _host(cn.view(g.ncell, 8), orig)
    return cn_h, orig_h, int(nspl.value)
