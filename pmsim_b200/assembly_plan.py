"""Host plan for assembling element blocks straight into the CSR values (no dense K_e round trip).

The element path writes every cell's dense element matrix and a second kernel gathers it into the
CSR values (the reference's ``GenericElement::kke`` followed by ``assemble_matrix``,
``src/fem/elements.rs:13-14``, ``src/base/assembly.rs:70-139``).  On meshes where the step is
memory-bound that round trip is most of the traffic.  Adding each cell's blocks straight into the
CSR values needs, per (cell, node a, node b), the CSR position of block (A, B), and an order of the
cells in which no two concurrent cells touch the same entry:

* ``color_cells``: a greedy colouring (cells of one colour share no node, so their blocks never
  meet); the sums then follow a fixed order, colour by colour, with no atomics;
* ``chunk_cells``: cells ordered along the longest axis and cut into chunks whose block rows fit a
  budget (sized to the L2 cache), each chunk sorted by colour, so that all colours of a chunk run
  back to back while its rows are cache-resident;
* ``block_slots``: for every cell and node pair, the index of block (A, B) in block row A.

This module holds the plan only; ``emulate`` applies it on the host to element matrices, which is
what the tests compare with the assembled matrix.
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh


def color_cells(mesh: Mesh) -> tuple[np.ndarray, int]:
    """Greedy colouring in cell order: each cell takes the smallest colour that no earlier cell
    sharing one of its nodes has.  Returns (colour of every cell, number of colours)."""
    used = np.zeros(mesh.npoint, dtype=np.uint64)  # bit k: a cell of colour k touches the node
    colors = np.empty(mesh.ncell, dtype=np.int32)
    for c, nodes in enumerate(mesh.cells):
        taken = np.bitwise_or.reduce(used[nodes])
        k = 0
        while (int(taken) >> k) & 1:
            k += 1
        if k >= 64:
            raise ValueError("more than 64 colours")
        colors[c] = k
        used[nodes] |= np.uint64(1 << k)
    return colors, int(colors.max()) + 1 if mesh.ncell else 0


def chunk_cells(mesh: Mesh, colors: np.ndarray, max_rows: int, axis: int | None = None):
    """Cells ordered along ``axis`` (default: the longest) by centroid and cut into chunks that touch
    at most ``max_rows`` block rows (nodes); inside a chunk the cells are sorted by colour (stable).
    Returns (order: the cells in execution order, chunk_ptr: chunk k is order[chunk_ptr[k]:
    chunk_ptr[k+1]], color_ptr: per chunk, the start of each colour, shape (nchunk, ncolor + 1))."""
    if axis is None:
        axis = int(np.argmax(np.ptp(mesh.coords, axis=0)))
    ncolor = int(colors.max()) + 1 if mesh.ncell else 0
    centroid = mesh.coords[mesh.cells, axis].mean(axis=1)
    by_pos = np.argsort(centroid, kind="stable")
    order, chunk_ptr, color_ptr = [], [0], []
    start = 0
    while start < len(by_pos):
        rows = set()
        end = start
        while end < len(by_pos):
            new = rows.union(mesh.cells[by_pos[end]].tolist())
            if len(new) > max_rows and end > start:
                break
            rows = new
            end += 1
        chunk = by_pos[start:end]
        chunk = chunk[np.argsort(colors[chunk], kind="stable")]
        order.extend(chunk.tolist())
        counts = np.bincount(colors[chunk], minlength=ncolor)
        color_ptr.append(np.concatenate([[0], np.cumsum(counts)]) + chunk_ptr[-1])
        chunk_ptr.append(chunk_ptr[-1] + len(chunk))
        start = end
    return np.array(order, dtype=np.int64), np.array(chunk_ptr, dtype=np.int64), np.array(color_ptr, dtype=np.int64)


def block_pattern(indptr: np.ndarray, indices: np.ndarray, ndim: int):
    """Block-row pointers and sorted block columns of a scalar CSR pattern of ndim x ndim node
    blocks (rows ndim*A .. ndim*A + ndim - 1 share the block columns of node A)."""
    npoint = (len(indptr) - 1) // ndim
    bptr = np.zeros(npoint + 1, dtype=np.int64)
    bcol = []
    for a in range(npoint):
        r = ndim * a
        cols = np.asarray(indices[indptr[r]:indptr[r + 1]])
        blocks = np.unique(cols // ndim)
        bcol.append(blocks)
        bptr[a + 1] = bptr[a] + len(blocks)
    return bptr, np.concatenate(bcol) if bcol else np.zeros(0, dtype=np.int64)


def block_slots(mesh: Mesh, bptr: np.ndarray, bcol: np.ndarray) -> np.ndarray:
    """slots[cell, a, b]: index of block (node a, node b) of the cell within block row conn[a]."""
    nn = mesh.nnode
    slots = np.empty((mesh.ncell, nn, nn), dtype=np.int32)
    for c, nodes in enumerate(mesh.cells):
        for a in range(nn):
            A = nodes[a]
            row = bcol[bptr[A]:bptr[A + 1]]
            k = np.searchsorted(row, nodes)
            if np.any(k >= len(row)) or np.any(row[np.minimum(k, len(row) - 1)] != nodes):
                raise ValueError(f"cell {c}: block row {A} of the pattern lacks a block of the cell")
            slots[c, a] = k
    return slots


def csr_position(bptr: np.ndarray, A: int, slot: int, i: int, j: int, ndim: int) -> int:
    """Position of entry (ndim*A + i, ndim*B + j) in the CSR values, B being block ``slot`` of row A
    (rows of a block row are stored one after another, each with all the row's block columns)."""
    nba = int(bptr[A + 1] - bptr[A])
    return int(ndim * ndim * bptr[A] + i * ndim * nba + slot * ndim + j)


def emulate(mesh: Mesh, ke: np.ndarray, bptr: np.ndarray, slots: np.ndarray, order: np.ndarray) -> np.ndarray:
    """The planned assembly on the host: every cell in ``order`` adds its element matrix
    ke[cell] (ne x ne) straight into the CSR values."""
    nd = mesh.ndim
    vals = np.zeros(int(nd * nd * bptr[-1]))
    for c in order:
        nodes = mesh.cells[c]
        for a, A in enumerate(nodes):
            for b in range(mesh.nnode):
                s = int(slots[c, a, b])
                for i in range(nd):
                    for j in range(nd):
                        vals[csr_position(bptr, int(A), s, i, j, nd)] += ke[c, a * nd + i, b * nd + j]
    return vals
