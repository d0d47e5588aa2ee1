"""CPU model of the on-chip simple update (dequantizer_b200/csrc/gates.cu,
simple_update_onchip_kernel), checked against the oracle's simple_update
(tensor_ops.py:265-389).

The kernel factors each side's matrix A[(b, o), (a, rho)] =
sum_i B[b, (a, i)] h[rho][o][i] in two Householder QRs (B = Q_B R_B, then
S = R_B h = Q_S R_S), builds the core from R_S of both sides, and forms
Gamma = (Q_B x I_o) Q_S [U; 0] / lambda with Q_B in compact-WY form
I - V T V^H (T from the reflectors as LAPACK's zlarft builds it). This model
runs exactly those steps in numpy (zgeqr2-convention reflectors, the same
index orders) and must reproduce the oracle's lambdas, truncation error,
entropy and two-site tensor to 1e-12 (FP64 on both sides).
"""

import numpy as np
import pytest

from oracle import tensor_ops as OT
from tests.helpers import two_site


def householder(A):
    """zgeqr2: returns (reflectors below the diagonal and R on/above it, tau)."""
    A = A.copy()
    m, n = A.shape
    k = min(m, n)
    tau = np.zeros(k, complex)
    for j in range(k):
        alpha = A[j, j]
        s = np.sum(np.abs(A[j + 1:, j]) ** 2)
        if s == 0.0 and alpha.imag == 0.0:
            continue
        beta = -np.copysign(np.sqrt(abs(alpha) ** 2 + s), alpha.real)
        tau[j] = complex((beta - alpha.real) / beta, -alpha.imag / beta)
        A[j + 1:, j] *= 1.0 / (alpha - beta)
        A[j, j] = beta
        v = np.concatenate([[1.0], A[j + 1:, j]])
        w = v.conj() @ A[j:, j + 1:]
        A[j:, j + 1:] -= np.conj(tau[j]) * np.outer(v, w)
    return A, tau


def vmat(F, k):
    m = F.shape[0]
    V = np.zeros((m, k), complex)
    for c in range(k):
        V[c, c] = 1.0
        V[c + 1:, c] = F[c + 1:, c]
    return V


def apply_q(F, tau, X):
    """X <- H_0 ... H_{k-1} X."""
    X = X.copy()
    V = vmat(F, len(tau))
    for j in range(len(tau) - 1, -1, -1):
        v = V[:, j]
        X -= tau[j] * np.outer(v, v.conj() @ X)
    return X


def zlarft(F, tau):
    k = len(tau)
    V = vmat(F, k)
    G = V.conj().T @ V
    T = np.zeros((k, k), complex)
    for j in range(k):
        T[:j, j] = T[:j, :j] @ (-tau[j] * G[:j, j])
        T[j, j] = tau[j]
    return V, T


def side(t, lams, half, slot, eps):
    """B, its QR, S and its QR for one side (lams: lambdas of every bond)."""
    k = t.ndim - 1
    d = t.shape[-1]
    others = [f for f in range(k) if f != slot]
    ce = t.shape[slot]
    tb = np.moveaxis(t, slot, -2)  # (others..., a, i)
    wt = np.ones(tb.shape[:-2])
    for n_, f in enumerate(others):
        wt = wt * lams[f].reshape([-1 if q == n_ else 1 for q in range(len(others))])
    B = (tb * wt[..., None, None]).reshape(-1, ce * d)  # rows b, columns (a, i)
    FB, tauB = householder(B)
    MB, KB = B.shape
    muB = min(MB, KB)
    RB = np.triu(FB[:muB])
    r = half.shape[0]
    # S[(c, o), (a, rho)] = sum_i R_B[c, (a, i)] h[rho][o][i]
    RB3 = RB.reshape(muB, ce, d)
    S = np.einsum("cai,roi->coar", RB3, half).reshape(muB * d, ce * r)
    S = S / np.linalg.norm(S)
    FS, tauS = householder(S)
    return dict(wt=wt, FB=FB, tauB=tauB, FS=FS, tauS=tauS, MB=MB, KB=KB, muB=muB, MS=muB * d, d=d, ce=ce, r=r,
                others=others, slot=slot, shape=t.shape)


def gamma(sd, X, rank, lams, eps):
    """(Q_B x I_o) Q_S X / lambda, back in the node tensor's index order."""
    d, muB = sd["d"], sd["muB"]
    Y = apply_q(sd["FS"], sd["tauS"], X)  # MS x rank
    Z = np.zeros((sd["MB"], d * rank), complex)
    Ytop = Y.reshape(muB, d, rank)  # rows (c, o)
    Z[:muB] = Ytop.transpose(0, 2, 1).reshape(muB, rank * d)  # columns q = col * d + o
    V, T = zlarft(sd["FB"], sd["tauB"])
    out = Z - V @ (T @ (V.conj().T @ Z))
    wt_inv = np.ones_like(sd["wt"])
    for n_, f in enumerate(sd["others"]):
        wt_inv = wt_inv * OT.safe_inverse(lams[f], eps).reshape(
            [-1 if q == n_ else 1 for q in range(len(sd["others"]))])
    shape_b = [sd["shape"][f] for f in sd["others"]]
    g = out.reshape(shape_b + [rank, d]) * wt_inv[..., None, None]
    return np.moveaxis(g, -2, sd["slot"])


def model_simple_update(t1, t2, l1, l2, h1, h2, i1, i2, eps, max_rank):
    s1 = side(t1, l1, h1, i1, eps)
    s2 = side(t2, l2, h2, i2, eps)
    K = s1["ce"] * s1["r"]
    mu, mv = min(s1["MS"], K), min(s2["MS"], K)
    Ru, Rv = np.triu(s1["FS"][:mu]), np.triu(s2["FS"][:mv])
    lam_e = np.repeat(l1[i1], s1["r"])
    core = (Ru * lam_e) @ Rv.T
    u, sv, vh = np.linalg.svd(core, full_matrices=False)
    sv = OT.safe_truncate(sv, eps)
    kk = min(mu, mv)
    rank = kk if max_rank is None else min(max_rank, kk)
    nrm = sv / np.linalg.norm(sv)
    ent = float(OT.entr(nrm**2).sum())
    err = float(np.linalg.norm(nrm[rank:]))
    Xu = np.zeros((s1["MS"], rank), complex)
    Xu[:mu] = u[:, :rank]
    Xv = np.zeros((s2["MS"], rank), complex)
    Xv[:mv] = vh[:rank].T
    return gamma(s1, Xu, rank, l1, eps), gamma(s2, Xv, rank, l2, eps), sv[:rank], err, ent


@pytest.mark.parametrize("chi,rank_gate,max_rank", [(4, 2, 4), (8, 2, 8), (16, 2, 16), (3, 4, 5), (16, 2, None)])
def test_onchip_simple_update_model_matches_oracle(chi, rank_gate, max_rank):
    rng = np.random.default_rng(chi + rank_gate)
    t1 = rng.standard_normal((chi, chi, chi, 2)) + 1j * rng.standard_normal((chi, chi, chi, 2))
    t2 = rng.standard_normal((chi, chi, chi, 2)) + 1j * rng.standard_normal((chi, chi, chi, 2))
    l1 = [np.sort(10 ** rng.uniform(-3, 0, chi))[::-1] for _ in range(3)]
    l2 = [l.copy() for l in l1[::-1]]
    l2[0] = l1[2].copy()
    if rank_gate == 2:
        gate = np.diag(np.exp(1j * rng.uniform(-3, 3, 4))).reshape(2, 2, 2, 2)
    else:
        q, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
        gate = q.reshape(2, 2, 2, 2)
    h1, h2 = OT.decompose_gate(gate, 1e-10)
    assert h1.shape[0] == rank_gate
    i1, i2 = 2, 0
    ref = OT.simple_update(t1.copy(), t2.copy(), l1, l2, h1, h2, i1, i2, 1e-10, None, max_rank)
    got = model_simple_update(t1, t2, l1, l2, h1, h2, i1, i2, 1e-10, max_rank)
    assert got[0].shape == ref[0].shape and got[1].shape == ref[1].shape
    assert np.abs(got[2] - ref[2]).max() < 1e-12 * ref[2].max()
    assert abs(got[3] - ref[3]) < 1e-12 and abs(got[4] - ref[4]) < 1e-12
    th_r = two_site(ref[0], ref[1], i1, i2, ref[2])
    th_g = two_site(got[0], got[1], i1, i2, got[2])
    assert np.abs(th_g - th_r).max() < 1e-12 * np.abs(th_r).max()
