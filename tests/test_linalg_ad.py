"""Hand-written spectral adjoints (dequantizer_b200.linalg_ad) on CPU.

Against torch's own backward on non-degenerate inputs with gauge-invariant
losses (functions of |U_ij|^2, |V_ij|^2 and the spectrum): 1e-12 relative.
On an exactly degenerate spectrum torch's backward divides by zero; the
broadened adjoints stay finite.
"""

import pytest
import torch

from dequantizer_b200.linalg_ad import eigh, product_svd, svd


@pytest.mark.parametrize("m,n", [(5, 5), (7, 4), (4, 7)])
def test_svd_adjoint_matches_torch(m, n):
    g = torch.Generator().manual_seed(m * 10 + n)
    A = torch.randn(3, m, n, dtype=torch.complex128, generator=g, requires_grad=True)
    k = min(m, n)
    wU = torch.randn(3, m, k, dtype=torch.float64, generator=g)
    wV = torch.randn(3, n, k, dtype=torch.float64, generator=g)
    wS = torch.randn(3, k, dtype=torch.float64, generator=g)

    M = torch.randn(3, m, n, dtype=torch.complex128, generator=g)
    wM = torch.randn(3, k, dtype=torch.float64, generator=g)

    def loss(fn):
        U, S, Vh = fn(A)
        # Re(u_j^H M v_j) is invariant only under the joint phase of (u_j, v_j),
        # so it exercises the phase term of the complex adjoint
        joint = torch.einsum("bij,bik,bjk->bk", M, U.conj(), Vh.mH).real
        return ((wU * U.abs() ** 2).sum() + (wV * Vh.mH.abs() ** 2).sum() + (wS * S).sum()
                + (wM * joint).sum())

    (g1,) = torch.autograd.grad(loss(lambda X: torch.linalg.svd(X, full_matrices=False)), A)
    (g2,) = torch.autograd.grad(loss(svd), A)
    assert float((g1 - g2).abs().max() / g1.abs().max()) < 1e-12


@pytest.mark.parametrize("m,n,K", [(8, 6, 4), (6, 9, 5), (5, 5, 8)])
def test_product_svd_adjoint_matches_torch(m, n, K):
    g = torch.Generator().manual_seed(m + n + K)
    X = torch.randn(m, K, dtype=torch.complex128, generator=g, requires_grad=True)
    Y = torch.randn(n, K, dtype=torch.complex128, generator=g, requires_grad=True)
    k = min(m, n, K)
    wU = torch.randn(m, k, dtype=torch.float64, generator=g)
    wW = torch.randn(n, k, dtype=torch.float64, generator=g)
    wS = torch.randn(k, dtype=torch.float64, generator=g)
    M = torch.randn(m, n, dtype=torch.complex128, generator=g)

    def loss(U, S, W):
        # Theta = U S W^T: the joint gauge is (u_j, w_j) -> (e^{i phi} u_j, e^{-i phi} w_j)
        joint = torch.einsum("ij,ik,jk->k", M, U.conj(), W.conj()).real
        return (wU * U.abs() ** 2).sum() + (wW * W.abs() ** 2).sum() + (wS * S).sum() + joint.sum()

    U, S, W = product_svd(X, Y)
    g1 = torch.autograd.grad(loss(U, S, W), (X, Y))
    U2, S2, Vh2 = torch.linalg.svd(X @ Y.T, full_matrices=False)
    U2, S2, W2 = U2[:, :k], S2[:k], Vh2[:k].T
    g2 = torch.autograd.grad(loss(U2, S2, W2), (X, Y))
    assert float((S - S2).abs().max()) < 1e-12
    for a, b in zip(g1, g2):
        assert float((a - b).abs().max() / b.abs().max()) < 1e-12


def test_eigh_adjoint_matches_torch():
    g = torch.Generator().manual_seed(1)
    H = torch.randn(3, 6, 6, dtype=torch.complex128, generator=g)
    H = (H + H.mH).requires_grad_(True)
    wV = torch.randn(3, 6, 6, dtype=torch.float64, generator=g)
    ww = torch.randn(3, 6, dtype=torch.float64, generator=g)

    def loss(fn):
        w, V = fn(H)
        return (wV * V.abs() ** 2).sum() + (ww * w).sum()

    (g1,) = torch.autograd.grad(loss(torch.linalg.eigh), H)
    (g2,) = torch.autograd.grad(loss(eigh), H)
    assert float((g1 - g2).abs().max() / g1.abs().max()) < 1e-12


def test_degenerate_spectra_stay_finite():
    # rank-2 4x4 matrix: two exactly zero singular values; identity: all equal eigenvalues
    a = torch.randn(4, 2, dtype=torch.complex128)
    A = (a @ a.mH).requires_grad_(True)
    U, S, Vh = svd(A)
    (gA,) = torch.autograd.grad((U.abs() ** 2 * torch.arange(4.0).unsqueeze(0)).sum() + S.sum(), A)
    assert torch.isfinite(gA).all()
    I = torch.eye(4, dtype=torch.complex128, requires_grad=True)
    w, V = eigh(I)
    (gI,) = torch.autograd.grad(w.sum() + (V.abs() ** 2).sum(), I)
    assert torch.isfinite(gI).all()


def test_product_svd_batched_equals_unbatched():
    g = torch.Generator().manual_seed(7)
    X = torch.randn(4, 9, 6, dtype=torch.complex128, generator=g, requires_grad=True)
    Y = torch.randn(4, 8, 6, dtype=torch.complex128, generator=g, requires_grad=True)
    M = torch.randn(4, 9, 8, dtype=torch.complex128, generator=g)

    def loss(U, S, W, M):
        return torch.einsum("...ij,...ik,...jk->...k", M, U.conj(), W.conj()).real.sum() + S.sum()

    gb = torch.autograd.grad(loss(*product_svd(X, Y), M), (X, Y))
    for b in range(4):
        gs = torch.autograd.grad(loss(*product_svd(X[b], Y[b]), M[b]), (X, Y))
        for a, c in zip(gb, gs):
            assert float((a[b] - c[b]).abs().max()) < 1e-12
