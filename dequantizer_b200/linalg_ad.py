"""SVD and Hermitian eigendecomposition with hand-written reverse passes.

The forward passes are torch.linalg (cuSOLVER on the GPU). The backward
passes are the standard spectral adjoints (complex case, torch's gradient
convention grad z = dL/dRe z + i dL/dIm z) with two guards that annealing
needs: exactly degenerate spectra occur there (zero singular values of
rank-deficient cores, equal Schmidt values by symmetry), so
  1 / (x_j - x_i)  ->  (x_j - x_i) / ((x_j - x_i)^2 + broadening)
  1 / s            ->  s / (s^2 + broadening)
(Lorentzian broadening). Away from degeneracies the result equals the exact
adjoint to within the broadening; inside a degenerate block the ill-defined
rotation terms are suppressed, which is exact for losses that do not depend
on the choice of basis inside the block (gauge-invariant ones).
"""

import torch

# The spectra differentiated here are O(1) (normalised two-site matrices,
# trace-1 messages): 1e-28 keeps gaps above ~1e-13 exact and damps
# rounding-level gaps (~1e-16), whose rotation terms are noise.
DEFAULT_BROADENING = 1e-28


def qr(X: torch.Tensor):
    """Reduced QR of a batch of matrices (..., m, k): the library's batched
    Householder kernel for complex128 tensors on the GPU (torch.linalg.qr
    elsewhere, e.g. CPU tests). Not differentiated."""
    if not (X.is_cuda and X.dtype == torch.complex128):
        return torch.linalg.qr(X, mode="reduced")
    from . import _lib

    m, k = X.shape[-2], X.shape[-1]
    kk = min(m, k)
    lead = X.shape[:-2]
    batch = 1
    for d in lead:
        batch *= int(d)
    A = X.detach().reshape(batch, m, k).contiguous()
    Q = torch.empty((batch, m, kk), dtype=X.dtype, device=X.device)
    R = torch.empty((batch, kk, k), dtype=X.dtype, device=X.device)
    nb = _lib.lib().dqz_qr_batched_scratch_bytes(batch, m, k)
    scratch = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=X.device)
    _lib.call("dqz_qr_batched", A.data_ptr(), batch, m, k, Q.data_ptr(), R.data_ptr(), scratch.data_ptr(),
              _lib.stream_handle())
    return Q.reshape(lead + (m, kk)), R.reshape(lead + (kk, k))


def _inv_lorentz(x: torch.Tensor, b: float) -> torch.Tensor:
    return x / (x * x + b)


def svd_adjoint(U, S, Vh, gU, gS, gVh, broadening: float, m: int, n: int) -> torch.Tensor:
    """Cotangent of A (m x n) from those of its SVD A = U diag(S) Vh, where U
    (m x k) and Vh (k x n) span the whole row and column spaces of A (thin
    SVD, or the SVD of a matrix of rank <= k)."""
    b = broadening
    k = S.shape[-1]
    V = Vh.mH
    cdt = U.dtype
    S2 = S * S
    E = S2.unsqueeze(-2) - S2.unsqueeze(-1)  # E_ij = s_j^2 - s_i^2
    F = _inv_lorentz(E, b)
    F.diagonal(dim1=-2, dim2=-1).zero_()
    Sinv = _inv_lorentz(S, b)
    inner = torch.zeros(U.shape[:-2] + (k, k), dtype=cdt, device=U.device)
    # phase term of the complex case: a loss invariant under the joint gauge
    # (u_j, v_j) -> e^{i phi} (u_j, v_j) has Im(u_j^H gU_j) = -Im(v_j^H gV_j);
    # the term is i Im(u_j^H gU_j - v_j^H gV_j) / (2 s_j)
    phase = torch.zeros(S.shape, dtype=S.dtype, device=S.device)
    if gU is not None:
        UhgU = U.mH @ gU
        inner = inner + (UhgU - UhgU.mH) * F * S.unsqueeze(-2)
        phase = phase + UhgU.diagonal(dim1=-2, dim2=-1).imag
    if gVh is not None:
        VhgV = V.mH @ gVh.mH
        inner = inner + S.unsqueeze(-1) * (VhgV - VhgV.mH) * F
        phase = phase - VhgV.diagonal(dim1=-2, dim2=-1).imag
    inner = inner + torch.diag_embed(1j * phase * Sinv / 2).to(cdt)
    if gS is not None:
        inner = inner + torch.diag_embed(gS.to(cdt))
    gA = U @ inner @ Vh
    if gU is not None and m > k:
        gUS = gU * Sinv.unsqueeze(-2)
        gA = gA + (gUS - U @ (U.mH @ gUS)) @ Vh
    if gVh is not None and n > k:
        SgVh = Sinv.unsqueeze(-1) * gVh
        gA = gA + U @ (SgVh - (SgVh @ V) @ Vh)
    return gA


class SVD(torch.autograd.Function):
    """A (..., m, n) -> (U, S, Vh), thin (k = min(m, n))."""

    @staticmethod
    def forward(ctx, A, broadening: float = DEFAULT_BROADENING):
        U, S, Vh = torch.linalg.svd(A, full_matrices=False)
        ctx.save_for_backward(U, S, Vh)
        ctx.broadening = broadening
        ctx.shape = A.shape
        return U, S, Vh

    @staticmethod
    def backward(ctx, gU, gS, gVh):
        U, S, Vh = ctx.saved_tensors
        gA = svd_adjoint(U, S, Vh, gU, gS, gVh, ctx.broadening, ctx.shape[-2], ctx.shape[-1])
        return gA, None


class ProductSVD(torch.autograd.Function):
    """SVD of Theta = X Y^T from its factors X (..., m, K), Y (..., n, K):
    Theta = U diag(S) W^T with U (m x k), W (n x k), k = min(m, n, K).

    Forward: X = Qx Rx, Y = Qy Ry (reduced QR), SVD of the core Rx Ry^T
    (the factorisation of tensor_ops.py:288 and :354-360). Backward: the SVD
    adjoint of Theta itself, Theta_bar formed explicitly, then
    X_bar = Theta_bar conj(Y), Y_bar = Theta_bar^T conj(X). The QR bases never
    enter the reverse pass, so neither their conditioning nor the basis
    freedom of degenerate factor spectra does (an SVD adjoint per factor
    would amplify rounding noise through 1 / (s_j^2 - s_i^2) terms of the
    factors' spectra that cancel only in exact arithmetic)."""

    @staticmethod
    def forward(ctx, X, Y, broadening: float = DEFAULT_BROADENING):
        Qx, Rx = qr(X)
        Qy, Ry = qr(Y)
        Uc, S, Vch = torch.linalg.svd(Rx @ Ry.mT, full_matrices=False)
        U = Qx @ Uc
        W = Qy @ Vch.mT
        ctx.save_for_backward(X, Y, U, S, W)
        ctx.broadening = broadening
        return U, S, W

    @staticmethod
    def backward(ctx, gU, gS, gW):
        X, Y, U, S, W = ctx.saved_tensors
        m, n = X.shape[-2], Y.shape[-2]
        Vh = W.mT  # Theta = U S W^T = U S Vh
        gVh = None if gW is None else gW.mT
        gT = svd_adjoint(U, S, Vh, gU, gS, gVh, ctx.broadening, m, n)
        return gT @ Y.conj(), gT.mT @ X.conj(), None


class EighH(torch.autograd.Function):
    """Hermitian A (..., n, n) -> (w ascending, V)."""

    @staticmethod
    def forward(ctx, A, broadening: float = DEFAULT_BROADENING):
        w, V = torch.linalg.eigh(A)
        ctx.save_for_backward(w, V)
        ctx.broadening = broadening
        return w, V

    @staticmethod
    def backward(ctx, gw, gV):
        w, V = ctx.saved_tensors
        cdt = V.dtype
        n = w.shape[-1]
        inner = torch.zeros(V.shape[:-2] + (n, n), dtype=cdt, device=V.device)
        if gV is not None:
            VhgV = V.mH @ gV
            sk = 0.5 * (VhgV - VhgV.mH)
            E = w.unsqueeze(-2) - w.unsqueeze(-1)  # E_ij = w_j - w_i
            F = _inv_lorentz(E, ctx.broadening)
            F.diagonal(dim1=-2, dim2=-1).zero_()
            inner = inner + sk * F
        if gw is not None:
            inner = inner + torch.diag_embed(gw.to(cdt))
        gA = V @ inner @ V.mH
        return gA, None


def svd(A, broadening: float = DEFAULT_BROADENING):
    return SVD.apply(A, broadening)


def product_svd(X, Y, broadening: float = DEFAULT_BROADENING):
    return ProductSVD.apply(X, Y, broadening)


def eigh(A, broadening: float = DEFAULT_BROADENING):
    return EighH.apply(A, broadening)
