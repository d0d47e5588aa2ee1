"""Two-site gate splitting, batched on the host (gate preparation, not the
hot path): the reference does the same 4x4 SVD per gate in
dequantizer/src/tensor_ops.py:202-218 (``_decompose_gate``).

A gate g[o1, o2, i1, i2] is regrouped as the (o1 i1) x (o2 i2) matrix,
decomposed G = U S V^H, and split into halves h1[r, o1, i1] = U[(o1 i1), r]
sqrt(S_r) and h2[r, o2, i2] = sqrt(S_r) V^H[r, (o2 i2)], keeping the singular
values above ``eps``.
"""

from typing import Tuple

import numpy as np

from . import _lib

HALF_SLOTS = 4  # gate rank r <= d1 * d1 = 4 for qubits


def decompose_gates(gates: np.ndarray, eps: float) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """gates: (n, d1, d2, d1, d2). Returns (halves, ranks, raw) where halves is
    (n, 2, 4, MAX_PHYS, MAX_PHYS) complex128 zero-padded in the layout the
    simple-update kernel reads (half j of gate n at halves[n, j], entries
    [rho, o, i] packed with stride d), and ranks is (n,) int32."""
    gates = np.asarray(gates, dtype=np.complex128)
    n, d1, d2 = gates.shape[0], gates.shape[1], gates.shape[2]
    if gates.shape[3] != d1 or gates.shape[4] != d2:
        raise ValueError("Input - output dimensions must match with each other.")
    if max(d1, d2) > _lib.MAX_PHYS:
        raise NotImplementedError("gate dimensions outside the supported range")
    mat = np.transpose(gates, (0, 1, 3, 2, 4)).reshape(n, d1 * d1, d2 * d2)
    u, s, vh = np.linalg.svd(mat, full_matrices=False)
    ranks = (s > eps).sum(axis=1).astype(np.int32)
    if ranks.max(initial=0) > HALF_SLOTS:
        raise NotImplementedError(f"gate rank above {HALF_SLOTS} is not supported")
    sq = np.sqrt(s)
    h1 = np.transpose((u * sq[:, None, :]).reshape(n, d1, d1, -1), (0, 3, 1, 2))  # (n, r, o1, i1)
    h2 = (vh * sq[:, :, None]).reshape(n, -1, d2, d2)  # (n, r, o2, i2)
    # zero the discarded ranks, then lay each half out as [rho][o][i] with
    # stride d from the start of its block of 4 * MAX_PHYS^2 entries
    keep = np.arange(h1.shape[1])[None, :] < ranks[:, None]
    mp = _lib.MAX_PHYS
    flat = np.zeros((n, 2, HALF_SLOTS * mp * mp), dtype=np.complex128)
    r_all = h1.shape[1]
    flat[:, 0, : r_all * d1 * d1] = (h1 * keep[:, :, None, None]).reshape(n, -1)
    flat[:, 1, : r_all * d2 * d2] = (h2 * keep[:, :, None, None]).reshape(n, -1)
    return flat, ranks, (h1, h2)


def decompose_gate(gate, eps: float):
    """Single gate (d1, d2, d1, d2) -> (controlling half (r, o1, i1), controlled half (r, o2, i2))."""
    g = np.asarray(gate, dtype=np.complex128)
    if g.ndim != 4:
        raise ValueError("Gate must be a tensor of rank 4.")
    _, ranks, (h1, h2) = decompose_gates(g[None], eps)
    r = int(ranks[0])
    return h1[0, :r], h2[0, :r]
