"""FP64 numpy restatement of dequantizer/src/tensor_ops.py.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke`` and
by ``bench.py``'s CPU-baseline leg as the checker. The product never imports it.

Each function follows the reference line by line (cited per function); LAPACK
comes from numpy's OpenBLAS build where the reference calls jax.numpy.linalg.
"""

from typing import List, Optional, Tuple, Union

import numpy as np

F32_MAX = float(np.finfo(np.float32).max)


def find_rank(lmbd: np.ndarray, accuracy: Optional[float], rank: Optional[int]) -> int:
    """tensor_ops.py:7-17 (also graph/tensor_utils.py:6-16)."""
    if accuracy is None:
        if rank is None:
            return int(lmbd.shape[0])
        return int(rank)
    scale = np.sqrt((lmbd**2).sum())
    return int(lmbd.shape[0] - (np.sqrt(np.cumsum(lmbd[::-1] ** 2)) / scale < accuracy).sum())


def safe_inverse(lmbd: np.ndarray, eps: float) -> np.ndarray:
    """tensor_ops.py:20-21."""
    return ((lmbd < eps) * F32_MAX + lmbd) ** -1


def safe_truncate(lmbd: np.ndarray, eps: float) -> np.ndarray:
    """tensor_ops.py:24-25."""
    return (lmbd > eps) * lmbd


def pass_through_node(tensor: np.ndarray, incoming: List[np.ndarray]) -> List[np.ndarray]:
    """tensor_ops.py:36-60: node -> edge messages from edge -> node messages.

    m_out_e[a', a] = sum conj(T)[.. a'_e ..] (T x_{f != e} m_f)[.. a_e ..],
    each message contracted over its second index, then divided by its trace."""
    degree = tensor.ndim - 1
    assert degree == len(incoming)
    conj_tensor = tensor.conj()
    out = []
    for idx in range(degree):
        up = tensor
        for i, message in enumerate(incoming):
            if i != idx:
                up = np.tensordot(up, message, axes=[0, 1])
            else:
                up = np.transpose(up, [*range(1, degree + 1), 0])
        up = np.transpose(up, [idx + 1, *range(idx + 1), *range(idx + 2, degree + 1)])
        down = np.transpose(conj_tensor, [idx, degree, *range(idx), *range(idx + 1, degree)])
        up = up.reshape((up.shape[0], -1))
        down = down.reshape((down.shape[0], -1))
        m = np.tensordot(down, up, axes=[1, 1])
        m = m / np.trace(m)
        out.append(m)
    return out


def pass_through_edge(incoming: List[np.ndarray]) -> List[np.ndarray]:
    """tensor_ops.py:70-76: an edge swaps its two incoming messages."""
    return [incoming[1], incoming[0]]


def absorb_by_node(tensor: np.ndarray, matrices: List[np.ndarray]) -> np.ndarray:
    """tensor_ops.py:88-93: contract each bond with a matrix's row index,
    cycle the physical index back to last, normalise."""
    for matrix in matrices:
        tensor = np.tensordot(tensor, matrix, axes=[0, 0])
    tensor = np.transpose(tensor, [*range(1, tensor.ndim), 0])
    return tensor / np.linalg.norm(tensor)


def edge_svd(incoming: List[np.ndarray], eps: float) -> Tuple[List[np.ndarray], np.ndarray]:
    """tensor_ops.py:108-130: Vidal orthogonalisers of one edge."""
    if len(incoming) != 2:
        raise NotImplementedError("Edge svd is not yet implemented for edge degrees != 2.")
    lf, uf = np.linalg.eigh(incoming[0])
    lb, ub = np.linalg.eigh(incoming[1])
    m_sq_inv_f = uf @ (np.sqrt(safe_inverse(lf, eps))[:, None] * uf.conj().T)
    m_sq_inv_b = ub @ (np.sqrt(safe_inverse(lb, eps))[:, None] * ub.conj().T)
    m_sq_f = uf @ (np.sqrt(safe_truncate(lf, eps))[:, None] * uf.conj().T)
    m_sq_b = ub @ (np.sqrt(safe_truncate(lb, eps))[:, None] * ub.conj().T)
    u, lmbd, vh = np.linalg.svd(np.tensordot(m_sq_f, m_sq_b, axes=[1, 1]), full_matrices=False)
    lmbd = lmbd / np.linalg.norm(lmbd)
    lmbd = safe_truncate(lmbd, eps)
    u = u * (lmbd > eps)[None]
    u = u / np.linalg.norm(u)
    vh = vh * (lmbd > eps)[:, None]
    vh = vh / np.linalg.norm(vh)
    return [m_sq_inv_f @ u, m_sq_inv_b @ vh.T], lmbd


def vidal_dist(tensor: np.ndarray, lambdas: List[np.ndarray], eps: float) -> float:
    """tensor_ops.py:143-175: sum over bonds of the trace norm of
    (normalised lambda^2-weighted reduced matrix - its ideal projector)."""
    degree = tensor.ndim - 1
    assert degree == len(lambdas)
    dist = 0.0
    conj_tensor = tensor.conj()
    for idx in range(degree):
        up = tensor.copy()
        for i, lmbd in enumerate(lambdas):
            if i == idx:
                continue
            up = up * lmbd.reshape(i * (1,) + (lmbd.shape[0],) + (degree - i) * (1,)) ** 2
        up = np.transpose(up, [idx, *range(idx), *range(idx + 1, degree + 1)])
        up = up.reshape((up.shape[0], -1))
        down = np.transpose(conj_tensor, [idx, *range(idx), *range(idx + 1, degree + 1)])
        down = down.reshape((down.shape[0], -1))
        result = np.tensordot(down, up, axes=[1, 1])
        result = result / np.trace(result)
        ideal = np.diag(np.diag(result).real > eps).astype(np.complex128)
        ideal = ideal / np.trace(ideal)
        dist += float(np.linalg.svd(result - ideal, compute_uv=False).sum())
    return dist


def canonicalize(tensor: np.ndarray, lambdas: List[np.ndarray], eps: float) -> np.ndarray:
    """tensor_ops.py:189-199: T * prod_e sqrt(truncated lambda_e), normalised."""
    degree = len(lambdas)
    assert degree == tensor.ndim - 1
    for idx, lmbd in enumerate(lambdas):
        lmbd = safe_truncate(lmbd.reshape(idx * (1,) + (lmbd.shape[0],) + (degree - idx) * (1,)), eps)
        tensor = tensor * np.sqrt(lmbd)
    return tensor / np.linalg.norm(tensor)


def decompose_gate(gate: np.ndarray, eps: float) -> Tuple[np.ndarray, np.ndarray]:
    """tensor_ops.py:202-218: SVD split of a (o1, o2, i1, i2) gate into halves
    (r, o1, i1) and (r, o2, i2) carrying sqrt of the kept singular values."""
    assert gate.ndim == 4 and gate.shape[0] == gate.shape[2] and gate.shape[1] == gate.shape[3]
    d1, d2 = gate.shape[0], gate.shape[1]
    g = np.transpose(gate, (0, 2, 1, 3)).reshape((d1 * d1, -1))
    u, lmbd, vh = np.linalg.svd(g, full_matrices=False)
    rank = int((lmbd > eps).sum())
    s = np.sqrt(lmbd[:rank])
    h1 = np.transpose((u[:, :rank] * s[None]).reshape((d1, d1, rank)), (2, 0, 1))
    h2 = (vh[:rank] * s[:, None]).reshape((rank, d2, d2))
    return h1, h2


def apply_half_gate(tensor: np.ndarray, half: np.ndarray, index: int) -> np.ndarray:
    """tensor_ops.py:221-237: contract the physical index with the half's
    input, merge the rank index into bond ``index`` (bond-major), normalise."""
    shape = list(tensor.shape)
    shape[index] *= half.shape[0]
    tensor = np.tensordot(tensor, half, axes=[-1, 2])
    n = tensor.ndim
    tensor = np.transpose(tensor, [*range(index + 1), n - 2, *range(index + 1, n - 2), n - 1])
    tensor = tensor.reshape(shape)
    return tensor / np.linalg.norm(tensor)


def apply_gate_halves(t1, t2, i1, i2, h1, h2):
    """tensor_ops.py:252-262."""
    return apply_half_gate(t1, h1, i1), apply_half_gate(t2, h2, i2)


def simple_update_preprocessing(tensor, lambdas, half, eps, index):
    """tensor_ops.py:265-295: lambda-scale the other bonds, apply the half gate,
    move bond ``index`` last, QR, undo the lambda scaling on Q."""
    degree = len(lambdas)
    assert tensor.ndim - 1 == degree
    for idx, lmbd in enumerate(lambdas):
        if idx == index:
            continue
        tensor = tensor * lmbd.reshape(idx * (1,) + (lmbd.shape[0],) + (degree - idx) * (1,))
    tensor = apply_half_gate(tensor, half, index)
    tensor = np.transpose(tensor, [*range(index), *range(index + 1, degree + 1), index])
    shape = tensor.shape
    q, r = np.linalg.qr(tensor.reshape((-1, shape[-1])))
    q = q.reshape((*shape[:-1], -1))
    others = [l for i, l in enumerate(lambdas) if i != index]
    for idx, lmbd in enumerate(others):
        q = q * safe_inverse(lmbd.reshape(idx * (1,) + (lmbd.shape[0],) + (degree - idx) * (1,)), eps)
    return q, r


def entr(x: np.ndarray) -> np.ndarray:
    """jax.scipy.special.entr: -x log x, 0 at 0, -inf below 0."""
    out = np.zeros_like(x)
    pos = x > 0
    out[pos] = -x[pos] * np.log(x[pos])
    out[x < 0] = -np.inf
    return out


def simple_update(t1, t2, lambdas1, lambdas2, h1, h2, i1, i2, eps, accuracy, max_rank=None):
    """tensor_ops.py:318-389. Returns (t1, t2, lambda, err, entropy)."""
    q1, r1 = simple_update_preprocessing(t1, lambdas1, h1, eps, i1)
    q2, r2 = simple_update_preprocessing(t2, lambdas2, h2, eps, i2)
    assert (np.abs(lambdas1[i1] - lambdas2[i2]) < 1e-5).all()
    lmbd_e = lambdas1[i1]
    additional = r1.shape[-1] // lmbd_e.shape[0]
    lmbd_e = np.tensordot(lmbd_e, np.ones((additional,)), axes=0).reshape((-1,))
    core = np.tensordot(r1 * lmbd_e, r2, axes=[1, 1])
    u, lmbd, vh = np.linalg.svd(core, full_matrices=False)
    lmbd = safe_truncate(lmbd, eps)
    rank = find_rank(lmbd, accuracy, max_rank)
    normalized = lmbd / np.linalg.norm(lmbd)
    entropy = float(entr(normalized**2).sum())
    err = float(np.linalg.norm(normalized[rank:]))
    lmbd = lmbd[:rank]
    u = u[:, :rank]
    vh = vh[:rank]
    t1 = np.tensordot(q1, u, axes=[-1, 0])
    d1 = t1.ndim - 1
    t2 = np.tensordot(q2, vh, axes=[-1, 1])
    d2 = t2.ndim - 1
    t1 = np.transpose(t1, [*range(i1), d1, *range(i1, d1)])
    t2 = np.transpose(t2, [*range(i2), d2, *range(i2, d2)])
    return t1, t2, lmbd, err, entropy
