"""Reference of the aggregation (block-Jacobi) preconditioner (test infrastructure only).

The checker for ktplace_b200/csrc/ktg_agg.cu: the same deterministic rules,
written as plain numpy / Python loops, so that the GPU's aggregates,
permutation and block inverses can be compared exactly on small systems.

The x and y systems are treated as one block-diagonal system of 2n rows
(row c < n is x row c, row c >= n is y row c - n); no entry couples the axes,
so no aggregate mixes them. Three levels of pairwise aggregation; the nodes
of level 0 are the rows of A (off-diagonal CSR, duplicates unmerged), a node
of level l + 1 is a matched pair or a single node of level l:

  dc(N): the node's Galerkin diagonal, the sum over its member rows m in
     position order of t_m = d_m + (m's entries whose column's node is N, in
     storage order); dc = d at level 0;
  strength of a stored entry (i, j, v) between the nodes A of i and B != A
     of j:  s = -v / sqrt(dc(A) * dc(B));
  ROUNDS handshake rounds: every unmatched node A picks the unmatched B
     with the largest s > 0 over all its member rows' entries (ties: smaller
     B); A and B are matched when they picked each other;
  leaders: unmatched nodes and the smaller node of each pair; the next
     level's ids number the leaders in order;
  fine row c follows its node: pos_c += size(a) when its node is b.

A node's coupling to another is its strongest single entry to it, so no
coarse matrix is formed.

Aggregates (at most 8 rows) are laid out contiguously in coarse-id order
(newpos = start of its aggregate + pos), which puts every x row before every
y row. Each aggregate's block of A (its rows and columns, duplicates summed)
is inverted in float64 by Cholesky; the preconditioner is that block-diagonal
inverse. A block whose Cholesky meets a non-positive pivot falls back to the
inverse of its diagonal.
"""
from __future__ import annotations

import numpy as np

ROUNDS = 2
LEVELS = 3
AGG_MAX = 1 << LEVELS


class _Level:
    """The fine rows: lists of (col, val) in storage order, and diag."""

    def __init__(self, cols, vals, diag):
        self.cols = cols
        self.vals = vals
        self.diag = diag


def _fine_level(sx: dict, sy: dict) -> _Level:
    n = sx["diag"].shape[0]
    cols, vals = [], []
    for off, s in ((0, sx), (n, sy)):
        rp = s["row_ptr"]
        for i in range(n):
            a, b = int(rp[i]), int(rp[i + 1])
            cols.append(s["col"][a:b].astype(np.int64) + off)
            vals.append(s["val"][a:b].astype(np.float64))
    return _Level(cols, vals, np.concatenate([sx["diag"], sy["diag"]]).astype(np.float64))


def _match(lv: _Level, cur: np.ndarray, dc: np.ndarray, N: int) -> np.ndarray:
    members = [[] for _ in range(N)]
    for c in range(cur.shape[0]):
        members[int(cur[c])].append(c)
    mate = np.full(N, -1, np.int64)
    for _ in range(ROUNDS):
        pick = np.full(N, -1, np.int64)
        for A in range(N):
            if mate[A] >= 0:
                continue
            best, bj = 0.0, -1
            for m in members[A]:
                for J, v in zip(lv.cols[m], lv.vals[m]):
                    B = int(cur[int(J)])
                    if B == A or mate[B] >= 0:
                        continue
                    s = -v / np.sqrt(dc[A] * dc[B])
                    if s > 0.0 and (s > best or (s == best and B < bj)):
                        best, bj = s, B
            pick[A] = bj
        for A in range(N):
            B = pick[A]
            if mate[A] < 0 and B >= 0 and pick[B] == A:
                mate[A] = B
    return mate


def _diagonals(lv: _Level, cur: np.ndarray, pos: np.ndarray, size: np.ndarray) -> np.ndarray:
    """dc of the nodes `cur` maps the rows to (positions pos, sizes size)."""
    R = cur.shape[0]
    t = np.empty(R)
    for c in range(R):
        acc = lv.diag[c]
        for J, v in zip(lv.cols[c], lv.vals[c]):
            if cur[int(J)] == cur[c]:
                acc = acc + v
        t[c] = acc
    mem = np.full((size.shape[0], AGG_MAX), -1, np.int64)
    mem[cur, pos] = np.arange(R)
    dc = np.empty(size.shape[0])
    for J in range(size.shape[0]):
        d = t[mem[J, 0]]
        for p in range(1, int(size[J])):
            d = d + t[mem[J, p]]
        dc[J] = d
    return dc


def aggregate(sx: dict, sy: dict) -> dict:
    """Aggregates of the combined system: agg id, position, start, newpos."""
    lv = _fine_level(sx, sy)
    R = lv.diag.shape[0]
    cur = np.arange(R, dtype=np.int64)
    pos = np.zeros(R, np.int64)
    size = np.ones(R, np.int64)
    dc = lv.diag.copy()
    N = R
    for level in range(LEVELS):
        mate = _match(lv, cur, dc, N)
        idx = np.arange(N)
        leader = (mate < 0) | (idx < mate)
        leaders = idx[leader]
        cid = np.empty(N, np.int64)
        cid[leaders] = np.arange(leaders.shape[0])
        cid[~leader] = cid[mate[~leader]]
        second = ~leader
        pos += np.where(second[cur], size[np.maximum(mate[cur], 0)], 0)
        new_size = size[leaders] + np.where(mate[leaders] >= 0, size[np.maximum(mate[leaders], 0)], 0)
        cur = cid[cur]
        size = new_size
        N = leaders.shape[0]
        if level + 1 < LEVELS:
            dc = _diagonals(lv, cur, pos, size)
    start = np.concatenate([[0], np.cumsum(size)])
    newpos = start[cur] + pos
    order = np.empty(R, np.int64)
    order[newpos] = np.arange(R)
    return {"agg": cur, "pos": pos, "size": size, "start": start, "newpos": newpos, "order": order}


def block_inverses(sx: dict, sy: dict, ag: dict) -> tuple:
    """minv[2n, 8] (row m of its block's inverse, by member offset) and meta
    (per-axis first row of the aggregate * 8 + size - 1), both in permuted order."""
    n = sx["diag"].shape[0]
    R = 2 * n
    minv = np.zeros((R, AGG_MAX))
    meta = np.zeros(R, np.int64)
    newpos = ag["newpos"]
    for J in range(ag["size"].shape[0]):
        first, k = int(ag["start"][J]), int(ag["size"][J])
        rows = ag["order"][first:first + k]
        axis = 1 if first >= n else 0
        s = sy if axis else sx
        B = np.zeros((k, k))
        for m, c in enumerate(rows):
            i = int(c) - axis * n
            B[m, m] += s["diag"][i]
            for e in range(int(s["row_ptr"][i]), int(s["row_ptr"][i + 1])):
                q = int(newpos[int(s["col"][e]) + axis * n]) - first
                if 0 <= q < k:
                    B[m, q] += s["val"][e]
        try:
            L = np.linalg.cholesky(B)
            Li = np.linalg.inv(L)
            inv = Li.T @ Li
        except np.linalg.LinAlgError:
            inv = np.diag(1.0 / np.diag(B))
        for m in range(k):
            minv[first + m, :k] = inv[m]
            meta[first + m] = (first - axis * n) * AGG_MAX + (k - 1)
    return minv, meta


def apply(minv: np.ndarray, meta: np.ndarray, r_perm: np.ndarray) -> np.ndarray:
    """u = M r in permuted order (both axes, 2n rows; meta is per axis)."""
    R = r_perm.shape[0]
    n = R // 2
    u = np.zeros(R)
    for c in range(R):
        axis = 1 if c >= n else 0
        first = int(meta[c] // AGG_MAX) + axis * n
        k = int(meta[c] % AGG_MAX) + 1
        u[c] = minv[c, :k] @ r_perm[first:first + k]
    return u
