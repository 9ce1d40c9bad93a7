"""CPU oracle of the predictor's configuration features (test infrastructure only).

Brute-force numpy restatement of vortexpasta.jl_b200/csrc/features.cu for small inputs (every
node is sampled): segment chords |x_i - x_prev(i)| (minimum image) and, per node, the nearest
quadrature point of a segment j with |j - i| > 2 and j != prev(i), capped at r_cut, binned over
log10(d / L) in 12 bins of width 1/4 from -3.  The features have no counterpart in the reference.
"""

from __future__ import annotations

import numpy as np


def minimum_image(d, L):
    return d - L * np.round(d / L)


def features(nodes, idx_prev, points, nquad, L, rcut):
    nodes = np.asarray(nodes, dtype=np.float64)
    Np = len(nodes)
    prev = np.asarray(idx_prev, dtype=np.int64)
    chords = np.linalg.norm(minimum_image(nodes - nodes[prev], L), axis=1)
    total = chords.sum()
    seg = np.arange(len(points)) // nquad
    hist = np.zeros(12)
    for i in range(Np):
        d = np.linalg.norm(minimum_image(nodes[i] - points, L), axis=1)
        keep = (np.abs(seg - i) > 2) & (seg != prev[i])
        best = min(rcut, d[keep].min()) if keep.any() else rcut
        b = int(np.floor((np.log10(best / L) + 3.0) * 4.0))
        hist[min(max(b, 0), 11)] += 1
    out = [np.log10(Np), np.log10(total / L**2), np.log10(total / Np / L), np.log10(chords[chords > 0].min() / L)]
    return np.concatenate([out, hist / Np])
