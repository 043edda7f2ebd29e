"""Synthetic H-matrices for layout tests (test helper).

Random quadtree partitions of an n_rows x n_cols point grid: each node splits
into four until a side reaches the leaf size or a coin says stop, so blocks
have unequal, non-power-of-two shapes.  Leaves are full rank or low rank
(rank 1 .. min(m, n) - 1) with N(0, 1) entries, a share `rank0_share` of the
low-rank leaves with rank 0 (no factors); both permutations are random.
Covers what BigWham's own cluster trees never produce: rectangular matrices
(source and receiver meshes of different sizes, BigWhamIO's rectangular
constructor, bigwham_io.h:85-96), odd block shapes and ragged ranks.
"""
import numpy as np

from oracle import HmatArrays


def _partition(r0, r1, c0, c1, rng, leaf, stop, out):
    if r1 - r0 <= leaf or c1 - c0 <= leaf or rng.random() < stop:
        out.append((r0, c0, r1, c1))
        return
    rm, cm = (r0 + r1) // 2, (c0 + c1) // 2
    for a, b in ((r0, rm), (rm, r1)):
        for c, d in ((c0, cm), (cm, c1)):
            _partition(a, b, c, d, rng, leaf, stop, out)


def synthetic_hmat(n_row_pts, n_col_pts, dof, seed, leaf=4, stop=0.25, lr_share=0.5,
                   rank0_share=0.0) -> HmatArrays:
    rng = np.random.default_rng(seed)
    blocks = []
    _partition(0, n_row_pts, 0, n_col_pts, rng, leaf, stop, blocks)
    fr, lr, fd, ld = [], [], [], []
    for i0, j0, i1, j1 in blocks:
        m, n = (i1 - i0) * dof, (j1 - j0) * dof
        if rng.random() >= lr_share or min(m, n) < 3:
            fr.append((i0, j0, i1, j1))
            fd.append(rng.standard_normal(m * n))
        else:
            r = int(rng.integers(1, min(m, n)))
            if rank0_share > 0 and rng.random() < rank0_share:
                r = 0
            lr.append((i0, j0, i1, j1, r))
            ld += [rng.standard_normal(m * r), rng.standard_normal(r * n)]
    cat = lambda a: np.concatenate(a) if a else np.zeros(0)  # noqa: E731
    return HmatArrays(dof, n_row_pts * dof, n_col_pts * dof, np.array(fr, np.int64).reshape(-1, 4),
                      np.array(lr, np.int64).reshape(-1, 5), cat(fd), cat(ld),
                      rng.permutation(n_row_pts).astype(np.int64), rng.permutation(n_col_pts).astype(np.int64))
