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
import torch

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


DIAG_SLOTS = ((0, 0), (0, 1), (1, 0), (1, 1))  # (rho, o) of the compact entries
# flat offsets of h[rho, o, o] in one half block ([rho][o][i], stride d = 2)
DIAG_FLAT_POS = np.array([(rho * 2 + o) * 2 + o for rho, o in DIAG_SLOTS], dtype=np.int64)


def decompose_diagonal_gates(diag, eps: float):
    """Split diagonal two-qubit gates g[o1,o2,i1,i2] = diag[o1,o2] d(o1,i1) d(o2,i2)
    (the annealing and Ising gates), vectorised over the batch, on the device
    ``diag`` lives on (a torch tensor, or a numpy array handled on the CPU).

    The regrouped (o1 i1) x (o2 i2) matrix is zero outside rows / columns
    (0,0) and (1,1), where it equals the 2x2 block A[o1][o2] = diag[o1, o2]; its
    SVD is that of A, done in closed form: V from the eigenvectors of A^H A,
    sigma_1 = sqrt(largest eigenvalue), sigma_2 = |det A| / sigma_1 (no
    cancellation, so the rank test sigma > eps matches a dense SVD), U = A V /
    sigma. Both halves are diagonal in (o, i), so only h[rho, o, o] is
    returned: compact (n, 2 halves, 4) complex128 with entries in
    ``DIAG_SLOTS`` order (zero for rho >= rank), and ranks (n,) int32, both of
    the input's kind. ``expand_diagonal_halves`` gives the layout of
    ``decompose_gates``."""
    as_numpy = not isinstance(diag, torch.Tensor)
    A = torch.as_tensor(np.asarray(diag) if as_numpy else diag).to(torch.complex128).reshape(-1, 2, 2)
    a, b, c, d = A[:, 0, 0], A[:, 0, 1], A[:, 1, 0], A[:, 1, 1]
    p = a.abs() ** 2 + c.abs() ** 2
    r = b.abs() ** 2 + d.abs() ** 2
    q = a.conj() * b + c.conj() * d
    lam1 = 0.5 * (p + r) + torch.sqrt(0.25 * (p - r) ** 2 + q.abs() ** 2)
    s1 = torch.sqrt(lam1)
    s2 = (a * d - b * c).abs() / torch.where(s1 > 0, s1, torch.ones_like(s1))
    # eigenvector of A^H A for lam1: (q, lam1 - p); a unit vector when q = 0
    # and lam1 = p (A^H A diagonal with the larger entry first)
    v0, v1 = q, (lam1 - p).to(torch.complex128)
    vn = torch.sqrt(v0.abs() ** 2 + v1.abs() ** 2)
    zero = vn < 1e-300
    first = (p >= r).to(torch.complex128)
    v0 = torch.where(zero, first, v0 / torch.where(zero, torch.ones_like(vn), vn))
    v1 = torch.where(zero, 1 - first, v1 / torch.where(zero, torch.ones_like(vn), vn))
    # V = [[v0, -conj(v1)], [v1, conj(v0)]] (columns = right singular vectors)
    V = torch.stack([torch.stack([v0, -v1.conj()], -1), torch.stack([v1, v0.conj()], -1)], -2)
    sig = torch.stack([s1, s2], -1)
    safe = torch.where(sig > 0, sig, torch.ones_like(sig))
    U = torch.einsum("nij,njr->nir", A, V) / safe[:, None, :]
    # second singular value zero: complete U orthonormally from its first column
    u2 = torch.stack([-U[:, 1, 0].conj(), U[:, 0, 0].conj()], -1)
    U = torch.stack([U[:, :, 0], torch.where((s2 > 0)[:, None], U[:, :, 1], u2)], -1)
    ranks = (sig > eps).sum(-1).to(torch.int32)
    sq = torch.sqrt(sig)
    cols = []
    for half in range(2):
        for rho, o in DIAG_SLOTS:
            keep = (rho < ranks).to(torch.float64)
            if half == 0:  # h1[rho, o, o] = U[o][rho] sqrt(s_rho)
                cols.append(U[:, o, rho] * sq[:, rho] * keep)
            else:  # h2[rho, o, o] = sqrt(s_rho) conj(V[o][rho])
                cols.append(sq[:, rho] * V[:, o, rho].conj() * keep)
    compact = torch.stack(cols, -1).reshape(-1, 2, 4)
    if as_numpy:
        return compact.numpy(), ranks.numpy()
    return compact, ranks


def expand_diagonal_halves(compact: np.ndarray) -> np.ndarray:
    """Compact diagonal halves (n, 2, 4) -> the zero-padded (n, 2, 4 * MAX_PHYS^2)
    layout of ``decompose_gates``."""
    n = compact.shape[0]
    mp = _lib.MAX_PHYS
    flat = np.zeros((n, 2, HALF_SLOTS * mp * mp), dtype=np.complex128)
    flat[:, :, DIAG_FLAT_POS] = compact
    return flat


def decompose_gate(gate, eps: float):
    """Single gate (d1, d2, d1, d2) -> (controlling half (r, o1, i1), controlled half (r, o2, i2))."""
    g = np.asarray(gate, dtype=np.complex128)
    if g.ndim != 4:
        raise ValueError("Gate must be a tensor of rank 4.")
    _, ranks, (h1, h2) = decompose_gates(g[None], eps)
    r = int(ranks[0])
    return h1[0, :r], h2[0, :r]
