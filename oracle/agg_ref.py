"""Reference of the aggregation (block-Jacobi) preconditioner (test infrastructure only).

The checker for ktplace_b200/csrc/ktg_agg.cu: the same deterministic rules,
written as plain numpy / Python loops, so that the GPU's aggregates,
permutation and block inverses can be compared exactly on small systems.

The x and y systems are treated as one block-diagonal system of 2n rows
(row c < n is x row c, row c >= n is y row c - n); no entry couples the axes,
so no aggregate mixes them. Three levels of pairwise aggregation:

  level 0 nodes are the rows of A (off-diagonal CSR, duplicates unmerged);
  strength of a stored entry (I, J, v):  s = -v / sqrt(d_I * d_J)
  ROUNDS handshake rounds: every unmatched node I picks the unmatched J != I
     with the largest s > 0 over its stored entries (ties: smaller J);
     I and J are matched when they picked each other;
  leaders: unmatched nodes and the smaller node of each pair; coarse ids
     number the leaders in order;
  coarse row of J = (a, b) (b = -1 if a is alone): the entries of row a, then
     of row b, mapped to coarse ids; entries mapping to J add to the coarse
     diagonal (d_a + entries(a -> J) + d_b + entries(b -> J), in that order),
     the others are summed per coarse id in that same (raw) order and stored
     with the ids ascending;
  fine row c follows its node: pos_c += size(a) when its node is b.

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
    """Rows of one level: lists of (col, val) in storage order, and diag."""

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


def _match(lv: _Level) -> np.ndarray:
    N = lv.diag.shape[0]
    d = lv.diag
    mate = np.full(N, -1, np.int64)
    for _ in range(ROUNDS):
        pick = np.full(N, -1, np.int64)
        for I in range(N):
            if mate[I] >= 0:
                continue
            best, bj = 0.0, -1
            for J, v in zip(lv.cols[I], lv.vals[I]):
                J = int(J)
                if J == I or mate[J] >= 0:
                    continue
                s = -v / np.sqrt(d[I] * d[J])
                if s > 0.0 and (s > best or (s == best and J < bj)):
                    best, bj = s, J
            pick[I] = bj
        for I in range(N):
            J = pick[I]
            if mate[I] < 0 and J >= 0 and pick[J] == I:
                mate[I] = J
    return mate


def _coarsen(lv: _Level, mate: np.ndarray, cid: np.ndarray, leaders: np.ndarray) -> _Level:
    cols, vals = [], []
    diag = np.zeros(leaders.shape[0])
    for J, a in enumerate(leaders):
        b = int(mate[a])
        sums: dict = {}
        dacc = lv.diag[a]
        for node in ((a, b) if b >= 0 else (a,)):
            if node == b:
                dacc = dacc + lv.diag[b]
            for col, v in zip(lv.cols[node], lv.vals[node]):
                K = int(cid[int(col)])
                if K == J:
                    dacc = dacc + v
                elif K in sums:
                    sums[K] = sums[K] + v
                else:
                    sums[K] = v
        diag[J] = dacc
        keys = sorted(sums)
        cols.append(np.array(keys, np.int64))
        vals.append(np.array([sums[k] for k in keys], np.float64))
    return _Level(cols, vals, diag)


def aggregate(sx: dict, sy: dict) -> dict:
    """Aggregates of the combined system: agg id, position, start, newpos."""
    lv = _fine_level(sx, sy)
    R = lv.diag.shape[0]
    cur = np.arange(R, dtype=np.int64)
    pos = np.zeros(R, np.int64)
    size = np.ones(R, np.int64)
    for level in range(LEVELS):
        mate = _match(lv)
        N = lv.diag.shape[0]
        idx = np.arange(N)
        leader = (mate < 0) | (idx < mate)
        leaders = idx[leader]
        cid = np.empty(N, np.int64)
        cid[leaders] = np.arange(leaders.shape[0])
        cid[~leader] = cid[mate[~leader]]
        second = ~leader
        pos += np.where(second[cur], size[np.maximum(mate[cur], 0)], 0)
        new_size = size[leaders] + np.where(mate[leaders] >= 0, size[np.maximum(mate[leaders], 0)], 0)
        if level + 1 < LEVELS:
            lv = _coarsen(lv, mate, cid, leaders)
        cur = cid[cur]
        size = new_size
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
