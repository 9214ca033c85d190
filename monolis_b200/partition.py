"""Row partition of a block-CSR system into rank-local systems with the halo
tables of MONOLIS_COM, the input layout of the reference's multi-rank solve
(each rank: its N owned block rows, then NP - N ghost rows whose values come
from their owners; recv/send tables list the local node ids exchanged with
every neighbour rank).

This stands in for the partitioner that produces those inputs in a monolis
application (the reference reads partitioned meshes written by its tools);
rows are split into contiguous ranges of about equal stored blocks."""
import numpy as np


def partition_rows(index, item, val, ndof, nranks):
    """index: N+1 offsets, item: 0-based block columns (ascending per row),
    val: blocks (nz * ndof^2). Returns one dict per rank with N, NP, the local
    CSR (index, 0-based item, val; ghost rows empty), glob (local -> global
    node ids) and the tables recv_pe, recv_index, recv_item, send_pe,
    send_index, send_item (0-based local node ids, neighbours ascending, each
    neighbour's list in ascending global id on both sides)."""
    index = np.asarray(index, dtype=np.int64)
    item = np.asarray(item, dtype=np.int64)
    val = np.asarray(val, dtype=np.float64)
    n = len(index) - 1
    b2 = ndof * ndof
    # contiguous row ranges with about equal stored blocks
    target = np.linspace(0, index[-1], nranks + 1)
    bounds = np.searchsorted(index, target[1:-1], side="left")
    bounds = np.concatenate([[0], np.maximum.accumulate(bounds), [n]]).astype(np.int64)
    owner = np.searchsorted(bounds, np.arange(n), side="right") - 1
    parts = []
    ghosts_of = []
    for r in range(nranks):
        lo, hi = int(bounds[r]), int(bounds[r + 1])
        cols = item[index[lo]:index[hi]]
        ghosts = np.unique(cols[(cols < lo) | (cols >= hi)])
        ghosts_of.append(ghosts)
        nown = hi - lo
        glob = np.concatenate([np.arange(lo, hi), ghosts])
        to_local = {int(g): i for i, g in enumerate(glob)}
        lidx = [0]
        litem = []
        lval = []
        for row in range(lo, hi):
            k0, k1 = index[row], index[row + 1]
            loc = np.array([to_local[int(c)] for c in item[k0:k1]], dtype=np.int64)
            order = np.argsort(loc, kind="stable")
            litem.append(loc[order])
            lval.append(val[k0 * b2:k1 * b2].reshape(-1, b2)[order].reshape(-1))
            lidx.append(lidx[-1] + (k1 - k0))
        lidx += [lidx[-1]] * len(ghosts)  # ghost rows: empty
        parts.append(dict(N=nown, NP=nown + len(ghosts), glob=glob, lo=lo, hi=hi,
                          index=np.array(lidx, dtype=np.int32),
                          item=np.concatenate(litem).astype(np.int32) if litem else np.zeros(0, np.int32),
                          val=np.concatenate(lval) if lval else np.zeros(0)))
    for r in range(nranks):
        p = parts[r]
        ghosts = ghosts_of[r]
        go = owner[ghosts] if len(ghosts) else np.zeros(0, dtype=np.int64)
        recv_pe, recv_index, recv_item = [], [0], []
        for s in sorted(set(go.tolist())):
            sel = np.nonzero(go == s)[0]  # ghosts are sorted by global id
            recv_pe.append(s)
            recv_item.extend((p["N"] + sel).tolist())
            recv_index.append(len(recv_item))
        send_pe, send_index, send_item = [], [0], []
        for s in range(nranks):
            if s == r:
                continue
            g = ghosts_of[s]
            mine = g[(g >= p["lo"]) & (g < p["hi"])]
            if len(mine) == 0:
                continue
            send_pe.append(s)
            send_item.extend((mine - p["lo"]).tolist())
            send_index.append(len(send_item))
        p.update(recv_pe=np.array(recv_pe, dtype=np.int32), recv_index=np.array(recv_index, dtype=np.int32),
                 recv_item=np.array(recv_item, dtype=np.int32), send_pe=np.array(send_pe, dtype=np.int32),
                 send_index=np.array(send_index, dtype=np.int32), send_item=np.array(send_item, dtype=np.int32))
    return parts


def partition_rank(index, item, val, ndof, nranks, rank):
    """partition_rows for one rank, vectorised (the C2 system has 56 M blocks):
    the same row ranges, local numbering (owned rows, then ghosts in
    ascending global id), per-row order of the local columns and halo
    tables, built with array operations. Returns that rank's dict."""
    index = np.asarray(index, dtype=np.int64)
    item = np.asarray(item)
    val = np.asarray(val, dtype=np.float64)
    n = len(index) - 1
    b2 = ndof * ndof
    target = np.linspace(0, index[-1], nranks + 1)
    bounds = np.searchsorted(index, target[1:-1], side="left")
    bounds = np.concatenate([[0], np.maximum.accumulate(bounds), [n]]).astype(np.int64)

    def ghosts_of(r):
        lo, hi = int(bounds[r]), int(bounds[r + 1])
        cols = item[index[lo]:index[hi]]
        return np.unique(cols[(cols < lo) | (cols >= hi)]).astype(np.int64)

    lo, hi = int(bounds[rank]), int(bounds[rank + 1])
    nown = hi - lo
    k0, k1 = int(index[lo]), int(index[hi])
    cols = item[k0:k1].astype(np.int64)
    outside = (cols < lo) | (cols >= hi)
    ghosts = np.unique(cols[outside])
    loc = np.where(outside, nown + np.searchsorted(ghosts, cols), cols - lo)
    rowid = np.repeat(np.arange(nown, dtype=np.int64), np.diff(index[lo:hi + 1]))
    order = np.lexsort((loc, rowid))
    lidx = np.concatenate([index[lo:hi + 1] - k0, np.full(len(ghosts), k1 - k0, dtype=np.int64)])
    part = dict(N=nown, NP=nown + len(ghosts), glob=np.concatenate([np.arange(lo, hi), ghosts]), lo=lo, hi=hi,
                index=lidx.astype(np.int32), item=loc[order].astype(np.int32),
                val=val[k0 * b2:k1 * b2].reshape(-1, b2)[order].reshape(-1))
    owner = np.searchsorted(bounds, ghosts, side="right") - 1
    recv_pe, counts = np.unique(owner, return_counts=True)  # ghosts ascending: owners grouped in order
    part.update(recv_pe=recv_pe.astype(np.int32),
                recv_index=np.concatenate([[0], np.cumsum(counts)]).astype(np.int32),
                recv_item=(nown + np.arange(len(ghosts))).astype(np.int32))
    send_pe, send_index, send_item = [], [0], []
    for s in range(nranks):
        if s == rank:
            continue
        g = ghosts_of(s)
        mine = g[(g >= lo) & (g < hi)]
        if len(mine) == 0:
            continue
        send_pe.append(s)
        send_item.append(mine - lo)
        send_index.append(send_index[-1] + len(mine))
    part.update(send_pe=np.array(send_pe, dtype=np.int32), send_index=np.array(send_index, dtype=np.int32),
                send_item=(np.concatenate(send_item) if send_item else np.zeros(0)).astype(np.int32))
    return part


def split_systems(nnz, nranks):
    """Independent systems (batched solve) over ranks, no communication:
    greedy longest-processing-time assignment by stored blocks -- systems in
    decreasing nnz order, each to the rank with the smallest load so far (ties
    to the lower rank). Returns one ascending list of system indices per rank;
    the largest load is at most 4/3 of the optimum (Graham's bound)."""
    nnz = np.asarray(nnz, dtype=np.int64)
    order = np.argsort(-nnz, kind="stable")
    load = np.zeros(nranks, dtype=np.int64)
    out = [[] for _ in range(nranks)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += nnz[i]
    return [sorted(o) for o in out]
