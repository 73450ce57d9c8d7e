"""Float32 numpy restatement of FeNNol's host graph builders (oracle; test-only).

``pair_list`` follows ``GraphGenerator.__call__``
(``src/fennol/models/preprocessing.py:74-355``):

* coordinates cast to float32 (``:81``);
* all pairs ``p1 < p2`` inside each system (``:106-119``);
* no cell: ``vec = x[p2] - x[p1]`` (``:121-123``);
* minimum image: ``s = -round(vec @ recip)``, ``vec += s @ cell``
  (``:127-143``; numpy ``round`` is half-to-even);
* general PBC: atoms wrapped with ``-floor(x @ recip)``, every image shift in
  ``[-n, n]^3`` with ``n = ceil(rc * |recip column|)`` (``:144-258``), and the
  stored shift is ``image + at_shift[p2] - at_shift[p1]`` (``:340-346``);
* ``d12 = (vec**2).sum(-1)`` -- numpy sums ``(x*x + y*y) + z*z`` -- kept
  when ``d12 < cutoff**2`` compared in float32 (``:264-266``).

The same numpy calls are used (``np.dot``, ``np.round``, ``np.floor``), so the
kept set equals the reference's.  Work is chunked to bound memory.

``filter_pairs`` restates ``GraphFilter.__call__`` (``:834-894``) and
``angular_triplets`` restates ``GraphAngularExtension.__call__``
(``:1085-1181``) as unordered edge pairs sharing a source.
"""

from __future__ import annotations

from typing import Dict, Optional

import numpy as np


def _chunks_upper_pairs(n: int, max_pairs: int = 4_000_000):
    """Yield (p1, p2) int64 arrays covering all i<j in [0, n), in row blocks."""
    i0 = 0
    while i0 < n - 1:
        # rows i0..i1-1 hold sum_{i}(n-1-i) pairs
        count = 0
        i1 = i0
        while i1 < n - 1 and count + (n - 1 - i1) <= max(max_pairs, n):
            count += n - 1 - i1
            i1 += 1
        rows = np.arange(i0, i1)
        lens = n - 1 - rows
        p1 = np.repeat(rows, lens)
        starts = np.repeat(np.cumsum(lens) - lens, lens)
        p2 = np.arange(p1.shape[0]) - starts + p1 + 1
        yield p1, p2
        i0 = i1


def pair_list(coordinates: np.ndarray, natoms, cells: Optional[np.ndarray] = None,
              reciprocal_cells: Optional[np.ndarray] = None, cutoff: float = 5.2,
              minimum_image: bool = True) -> Dict[str, np.ndarray]:
    """All pairs ``p1 < p2`` (global atom indices) with ``d12 < cutoff**2``.

    ``cells``/``reciprocal_cells``: ``[B,3,3]`` or ``[1,3,3]`` (one cell for all
    systems), rows are lattice vectors.  Returns sorted ``p1, p2, shift[int,3],
    d12[float32]``.
    """
    coords = np.array(coordinates, dtype=np.float32)
    natoms = np.asarray(natoms, dtype=np.int64).reshape(-1)
    offsets = np.concatenate([[0], np.cumsum(natoms)])
    apply_pbc = cells is not None
    if apply_pbc:
        if reciprocal_cells is None:
            # the reference inverts the caller's cells in their own precision
            # (check_input, preprocessing.py:1780-1781) and casts the result to
            # float32 in the builder (:126)
            reciprocal_cells = np.linalg.inv(np.asarray(cells).reshape(-1, 3, 3))
        cells = np.array(cells, dtype=np.float32).reshape(-1, 3, 3)
        recips = np.array(reciprocal_cells, dtype=np.float32).reshape(-1, 3, 3)
    rc2 = cutoff ** 2
    out_p1, out_p2, out_s, out_d = [], [], [], []
    for b in range(natoms.shape[0]):
        off, n = int(offsets[b]), int(natoms[b])
        if n < 2:
            continue
        x = coords[off:off + n]
        if apply_pbc:
            cell = cells[b if cells.shape[0] > 1 else 0]
            recip = recips[b if recips.shape[0] > 1 else 0]
            if not minimum_image:
                at_shifts = -np.floor(np.dot(x, recip))
                x = x + np.dot(at_shifts, cell)
                inv_d = np.sum(recip ** 2, axis=0) ** 0.5
                nrep = np.ceil(np.float32(cutoff) * inv_d).astype(np.int64)
                grid = np.array(np.meshgrid(*[np.arange(-k, k + 1) for k in nrep]),
                                dtype=np.float32).T.reshape(-1, 3)
                dvec = np.dot(grid, cell)
        for p1, p2 in _chunks_upper_pairs(n):
            vec = x[p2] - x[p1]
            if not apply_pbc:
                d12 = (vec ** 2).sum(axis=-1)
                keep = d12 < rc2
                shifts = np.zeros((int(keep.sum()), 3))
                q1, q2, dd = p1[keep], p2[keep], d12[keep]
            elif minimum_image:
                s = -np.round(np.dot(vec, recip))
                vec = vec + np.dot(s, cell)
                d12 = (vec ** 2).sum(axis=-1)
                keep = d12 < rc2
                q1, q2, dd, shifts = p1[keep], p2[keep], d12[keep], s[keep]
            else:
                v = (vec[:, None, :] + dvec[None, :, :])
                d12 = (v ** 2).sum(axis=-1)
                keep = d12 < rc2
                pi, si = np.nonzero(keep)
                q1, q2, dd = p1[pi], p2[pi], d12[pi, si]
                shifts = grid[si] + at_shifts[q2] - at_shifts[q1]
            out_p1.append(q1 + off)
            out_p2.append(q2 + off)
            out_s.append(np.asarray(shifts).reshape(-1, 3))
            out_d.append(dd.astype(np.float32))
    if out_p1:
        p1 = np.concatenate(out_p1)
        p2 = np.concatenate(out_p2)
        sh = np.rint(np.concatenate(out_s)).astype(np.int64)
        d12 = np.concatenate(out_d)
    else:
        p1 = p2 = np.zeros(0, np.int64)
        sh = np.zeros((0, 3), np.int64)
        d12 = np.zeros(0, np.float32)
    order = np.lexsort((sh[:, 2], sh[:, 1], sh[:, 0], p2, p1))
    return {"p1": p1[order], "p2": p2[order], "shift": sh[order], "d12": d12[order]}


def filter_pairs(pairs: Dict[str, np.ndarray], cutoff: float) -> Dict[str, np.ndarray]:
    """Sub-list with ``d12 < cutoff**2`` (``GraphFilter.__call__``, ``:854-866``;
    also the skin-to-cutoff step ``:295-318``)."""
    keep = np.asarray(pairs["d12"], dtype=np.float32) < cutoff ** 2
    return {k: v[keep] for k, v in pairs.items()}


def symmetrize(pairs: Dict[str, np.ndarray]):
    """Directed edges ``src=[p1,p2], dst=[p2,p1], shift=[s,-s]`` (``:320-326``)."""
    src = np.concatenate([pairs["p1"], pairs["p2"]])
    dst = np.concatenate([pairs["p2"], pairs["p1"]])
    sh = np.concatenate([pairs["shift"], -pairs["shift"]])
    d12 = np.concatenate([pairs["d12"], pairs["d12"]])
    return src, dst, sh, d12


def angular_triplets(edge_src: np.ndarray, nat: int):
    """Unordered pairs of directed edges with the same source
    (``GraphAngularExtension.__call__``, ``:1085-1181``).

    Returns ``angle_src, angle_dst`` (edge indices, ``angle_src`` listed first
    in source-sorted order) and ``central_atom``.
    """
    edge_src = np.asarray(edge_src, dtype=np.int64)
    if edge_src.size == 0:
        z = np.zeros(0, np.int64)
        return z, z, z
    order = np.argsort(edge_src, kind="stable")
    srt = edge_src[order]
    count = np.bincount(srt, minlength=nat)
    max_count = int(count.max())
    starts = np.concatenate([[0], np.cumsum(count)[:-1]])
    local = np.arange(srt.shape[0]) - starts[srt]
    table = np.full((nat, max_count), -1, dtype=np.int64)
    table[srt, local] = order
    a, b = np.triu_indices(max_count, 1)
    asrc = table[:, a].ravel()
    adst = table[:, b].ravel()
    valid = (asrc >= 0) & (adst >= 0)
    asrc, adst = asrc[valid], adst[valid]
    return asrc, adst, edge_src[asrc]


def canonical_from_ell(nbr_j: np.ndarray, nbr_shift: np.ndarray, nbr_count: np.ndarray):
    """Turn per-atom neighbour rows (j, shift) into the reference's canonical
    half list ``p1 < p2`` sorted like :func:`pair_list`, and check that every
    row entry has its mirror ``(j, i, -s)``.  Returns (dict, symmetric: bool)."""
    n = nbr_count.shape[0]
    cnt = np.minimum(nbr_count, nbr_j.shape[1])
    rows = np.repeat(np.arange(n), cnt)
    cols = np.concatenate([np.arange(c) for c in cnt]) if n else np.zeros(0, np.int64)
    j = nbr_j[rows, cols].astype(np.int64)
    s = nbr_shift[rows, cols].astype(np.int64).reshape(-1, 3)
    fwd = np.stack([rows, j, s[:, 0], s[:, 1], s[:, 2]], 1)
    rev = np.stack([j, rows, -s[:, 0], -s[:, 1], -s[:, 2]], 1)
    fs = {tuple(r) for r in fwd.tolist()}
    rs = {tuple(r) for r in rev.tolist()}
    symmetric = fs == rs and len(fs) == fwd.shape[0]
    half = fwd[fwd[:, 0] < fwd[:, 1]]
    order = np.lexsort((half[:, 4], half[:, 3], half[:, 2], half[:, 1], half[:, 0]))
    half = half[order]
    return {"p1": half[:, 0], "p2": half[:, 1], "shift": half[:, 2:5]}, symmetric
