"""CPU model of the data flow of the tcgen05 node update (dequantizer_b200/csrc/bp_umma.cu).

The kernel's correctness rests on index formulas: the two BF16 core-matrix
layouts of a node tensor, the shared-memory layouts its TMEM readback writes,
the UMMA shared-memory descriptors (start, leading / stride byte offsets,
K- or MN-major, no swizzle) through which the tensor cores read operands, and
the ldmatrix addresses of the final warp-level products. This test restates
those formulas (same constants as the kernel) and runs the kernel's sequence
of operations on numpy arrays:

* every operand the tensor cores read is fetched through a model of the
  no-swizzle canonical layout: element (m, k) of a K-major operand at byte
  start + (m/8)*SBO + (k/8)*LBO + (m%8)*16 + (k%8)*2, of an MN-major one at
  start + (m/8)*SBO + (k/8)*LBO + (k%8)*16 + (m%8)*2;
* every complex product is the kernel's pair of real products, the real
  plane against [Re m^T | Im m^T] and the imaginary plane against
  [-Im m^T | Re m^T], with 32 accumulator columns Re | Im;
* the final products read 8 x 8 matrices at the kernel's ldmatrix row
  addresses.

In FP64 the modelled messages equal the oracle's pass_through_node
(tensor_ops.py:36-60) to rounding; with BF16 rounding at the points where the
kernel rounds (inputs, stage-1 and stage-2 outputs) they stay within the
3e-2 bound the GPU tests use.
"""

import numpy as np
import pytest

from oracle import tensor_ops as OT

PLANE = 4096
XS_SBO, XS_L = 72, 32 * 72
Y_AS = 264


def off_l1(a, b, c):
    return ((c * 2 + (a >> 3)) * 2 + (b >> 3)) * 64 + (a & 7) * 8 + (b & 7)


def off_l2(a, b, c):
    return ((a * 2 + (b >> 3)) * 2 + (c >> 3)) * 64 + (b & 7) * 8 + (c & 7)


def bf16(x):
    """Round float64 values to BF16 (nearest, ties to even) and back."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def umma_read(plane, start_el, lbo_b, sbo_b, rows, mn_major):
    """Operand (rows x 16) read by a tcgen05 MMA from a no-swizzle layout."""
    m = np.arange(rows)[:, None]
    k = np.arange(16)[None, :]
    if mn_major:
        byte = (m // 8) * sbo_b + (k // 8) * lbo_b + (k % 8) * 16 + (m % 8) * 2
    else:
        byte = (m // 8) * sbo_b + (k // 8) * lbo_b + (m % 8) * 16 + (k % 8) * 2
    assert np.all(byte % 2 == 0)
    return plane[start_el + byte // 2]


def b_planes(msg, rnd):
    """The two K-major message operands (32 n x 16 k): [Re m^T | Im m^T] and
    [-Im m^T | Re m^T], element (k, n) at ((n/8)*2 + k/8)*64 + (n%8)*8 + k%8."""
    br, bi = np.zeros(512), np.zeros(512)
    for n in range(16):
        for k in range(16):
            lo = ((n >> 3) * 2 + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7)
            hi = (((n + 16) >> 3) * 2 + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7)
            br[lo], br[hi] = rnd(msg[n, k].real), rnd(msg[n, k].imag)
            bi[lo], bi[hi] = rnd(-msg[n, k].imag), rnd(msg[n, k].real)
    return br, bi


def mma_tile(a_re, a_im, a_start, a_lbo, a_sbo, a_mn, b):
    """One 128-row tile: D (128 x 32) = A_re . B_r + A_im . B_i."""
    br, bi = b
    Br = umma_read(br, 0, 128, 256, 32, False)  # (n, k)
    Bi = umma_read(bi, 0, 128, 256, 32, False)
    Ar = umma_read(a_re, a_start, a_lbo, a_sbo, 128, a_mn)
    Ai = umma_read(a_im, a_start, a_lbo, a_sbo, 128, a_mn)
    return Ar @ Br.T + Ai @ Bi.T


def store_row(re, im, val, off, rnd):
    for h in range(2):
        o = off(h)
        re[o:o + 8] = rnd(val[8 * h:8 * h + 8])
        im[o:o + 8] = rnd(val[16 + 8 * h:16 + 8 * h + 8])


def frag(plane, core):
    """16 x 16 fragment of four 8 x 8 matrices i = 0..3 (rows i&1, cols i>>1):
    row r of matrix i at core(i) + r*8."""
    f = np.zeros((16, 16))
    for i in range(4):
        for r in range(8):
            f[(i & 1) * 8 + r, (i >> 1) * 8:(i >> 1) * 8 + 8] = plane[core(i) + r * 8:core(i) + r * 8 + 8]
    return f


def frag_b_rows(plane, core):
    """B (k x n = 16 x 16) from matrices stored [n rows][k contiguous]:
    matrix i = (n-tile i>>1, k-half i&1)."""
    b = np.zeros((16, 16))
    for i in range(4):
        blk = plane[core(i):core(i) + 64].reshape(8, 8)  # [n][k]
        b[(i & 1) * 8:(i & 1) * 8 + 8, (i >> 1) * 8:(i >> 1) * 8 + 8] = blk.T
    return b


def frag_b_trans(plane, core):
    """B (k x n) from matrices stored [k rows][n contiguous]: matrix i =
    (k-half i&1, n-tile i>>1)."""
    b = np.zeros((16, 16))
    for i in range(4):
        blk = plane[core(i):core(i) + 64].reshape(8, 8)  # [k][n]
        b[(i & 1) * 8:(i & 1) * 8 + 8, (i >> 1) * 8:(i >> 1) * 8 + 8] = blk
    return b


def model_node_update(T, msgs, rnd):
    """Messages of the three bonds as the kernel computes them (T: (16,16,16,2))."""
    B = [b_planes(m, rnd) for m in msgs]
    out = [np.zeros((16, 16), complex) for _ in range(3)]
    idx = np.arange(16)
    a, b, c = np.meshgrid(idx, idx, idx, indexing="ij")
    for s in range(2):
        L1r, L1i, L2r, L2i = (np.zeros(PLANE) for _ in range(4))
        ts = T[..., s]
        L1r[off_l1(a, b, c)], L1i[off_l1(a, b, c)] = rnd(ts.real), rnd(ts.imag)
        L2r[off_l2(a, b, c)], L2i[off_l2(a, b, c)] = rnd(ts.real), rnd(ts.imag)
        XSr, XSi = np.zeros(2 * XS_L), np.zeros(2 * XS_L)
        XS2r, XS2i, XPr, XPi = (np.zeros(PLANE) for _ in range(4))
        for t in range(2):
            D1 = mma_tile(L1r, L1i, 64 * t, 256, 512, True, B[0])       # X = T x_0 m0
            Dp = mma_tile(L2r, L2i, 2048 * t, 128, 256, False, B[2])    # X" = T x_2 m2
            for m in range(128):
                cc, bl = m >> 3, m & 7
                store_row(XSr, XSi, D1[m], lambda ah: (cc >> 3) * XS_L + ((t * 2 + ah) * 8 + bl) * XS_SBO
                          + (cc & 7) * 8, rnd)
                store_row(XS2r, XS2i, D1[m], lambda ah: t * 2048 + (cc * 2 + ah) * 64 + bl * 8, rnd)
                aa, bb = 8 * t + (m >> 4), m & 15
                store_row(XPr, XPi, Dp[m], lambda ch: (bb >> 3) * 2048 + (aa * 2 + ch) * 64 + (bb & 7) * 8, rnd)
        Y1r, Y1i, Y2r, Y2i, Y0r, Y0i = (np.zeros(16 * Y_AS) for _ in range(6))
        for t in range(2):
            D2 = mma_tile(XSr, XSi, t * 16 * XS_SBO, XS_L * 2, XS_SBO * 2, True, B[2])   # Y1 = X x_2 m2
            D3 = mma_tile(XS2r, XS2i, 1024 * t, 4096, 128, True, B[1])                 # Y2 = X x_1 m1
            D5 = mma_tile(XPr, XPi, 1024 * t, 4096, 128, True, B[1])                   # Y0 = X" x_1 m1
            for m in range(128):
                ap, bl = (m >> 6) * 8 + (m & 7), (m >> 3) & 7
                store_row(Y1r, Y1i, D2[m], lambda ch: ap * Y_AS + (t * 2 + ch) * 64 + bl * 8, rnd)
                ap2, cl = m & 15, m >> 4
                store_row(Y2r, Y2i, D3[m], lambda bh: ap2 * Y_AS + (t * 2 + bh) * 64 + cl * 8, rnd)
                cp, al = m & 15, m >> 4
                store_row(Y0r, Y0i, D5[m], lambda bh: cp * Y_AS + (t * 2 + bh) * 64 + al * 8, rnd)
        for j in range(16):  # K-steps (a' for out_1 and out_2, c' for out_0)
            ya = lambda i: j * Y_AS + ((i & 1) * 2 + (i >> 1)) * 64
            l1_rows = lambda i: ((j * 2 + (i >> 1)) * 2 + (i & 1)) * 64
            l2_rows = lambda i: ((j * 2 + (i >> 1)) * 2 + (i & 1)) * 64
            l2_trans = lambda i: ((j * 2 + (i & 1)) * 2 + (i >> 1)) * 64
            for e, (Yr, Yi, Lr, Li, fb, core) in enumerate([
                    (Y0r, Y0i, L1r, L1i, frag_b_rows, l1_rows),
                    (Y1r, Y1i, L2r, L2i, frag_b_rows, l2_rows),
                    (Y2r, Y2i, L2r, L2i, frag_b_trans, l2_trans)]):
                A = frag(Yr, ya) + 1j * frag(Yi, ya)
                Bm = fb(Lr, core) + 1j * fb(Li, core)
                out[e] += A @ np.conj(Bm)
    return [o.T / np.trace(o) for o in out]  # message[n][m] = out_e[m][n] / trace


def _inputs(seed):
    rng = np.random.default_rng(seed)
    T = (rng.standard_normal((16, 16, 16, 2)) + 1j * rng.standard_normal((16, 16, 16, 2))) / 64
    msgs = []
    for _ in range(3):
        a = rng.standard_normal((16, 16)) + 1j * rng.standard_normal((16, 16))
        m = a @ a.conj().T
        msgs.append(m / np.trace(m).real)
    return T, msgs


def test_umma_layout_model_matches_oracle_fp64():
    T, msgs = _inputs(3)
    got = model_node_update(T, msgs, lambda x: np.asarray(x, dtype=np.float64))
    ref = OT.pass_through_node(T, msgs)
    for e in range(3):
        assert np.abs(got[e] - ref[e]).max() < 1e-12 * np.abs(ref[e]).max()


@pytest.mark.parametrize("seed", [4, 5])
def test_umma_layout_model_bf16_error_bound(seed):
    T, msgs = _inputs(seed)
    got = model_node_update(T, msgs, bf16)
    ref = OT.pass_through_node(T, msgs)
    for e in range(3):
        err = np.abs(got[e] - ref[e]).max() / np.abs(ref[e]).max()
        assert 1e-5 < err < 3e-2


def test_umma_layout_model_matches_reference_golden():
    """The modelled kernel data flow on the reference's own recorded
    pass_through_node at this shape (tests/golden, degree 3, bonds 16)."""
    import os

    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tensor_ops_golden.npz"))
    T = g["ptn_k3_chi16/tensor"]
    msgs = [g[f"ptn_k3_chi16/msg{i}"] for i in range(3)]
    got = model_node_update(T, msgs, lambda x: np.asarray(x, dtype=np.float64))
    for e in range(3):
        ref = g[f"ptn_k3_chi16/out{e}"]
        assert np.abs(got[e] - ref).max() < 1e-12 * np.abs(ref).max()
