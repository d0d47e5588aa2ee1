"""The oracle against golden vectors of the reference's own tensor_ops.

tests/golden/tensor_ops_golden.npz holds inputs and outputs of the
reference's hot-path functions (dequantizer/src/tensor_ops.py), computed by
running the reference module itself (tests/golden/make_golden.py; numpy
standing in for jax.numpy). Each oracle function must reproduce them: node
updates, edge SVDs (orthogonalisers and lambdas), absorption, Vidal distance,
canonicalisation, gate decomposition, half-gate application and the simple
update, including a rank-deficient edge and both truncation rules.
"""

import os

import numpy as np
import pytest

from oracle import tensor_ops as OT

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tensor_ops_golden.npz")
TOL = 1e-12


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLDEN))


def lst(g, key):
    return [g[f"{key}{i}"] for i in range(int(g[f"{key}_n"]))]


def close(a, b, tol=TOL):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    scale = max(np.abs(b).max(), 1e-300)
    assert np.abs(a - b).max() <= tol * scale


@pytest.mark.parametrize("case", ["ptn_k2", "ptn_k3", "ptn_k4", "ptn_k3_d3", "ptn_k3_chi16"])
def test_pass_through_node(g, case):
    out = OT.pass_through_node(g[f"{case}/tensor"], lst(g, f"{case}/msg"))
    for a, b in zip(out, lst(g, f"{case}/out")):
        close(a, b)


@pytest.mark.parametrize("case", ["esvd_full", "esvd_def"])
def test_edge_svd(g, case):
    orth, lam = OT.edge_svd(lst(g, f"{case}/msg"), 1e-10)
    close(lam, g[f"{case}/lam"])
    for a, b in zip(orth, lst(g, f"{case}/orth")):
        close(a, b, 1e-10)


def test_absorb_by_node(g):
    close(OT.absorb_by_node(g["abs_k3/tensor"], lst(g, "abs_k3/mat")), g["abs_k3/out"])


def test_vidal_dist_and_canonicalize(g):
    lams = lst(g, "vd_k3/lam")
    close(OT.vidal_dist(g["vd_k3/tensor"], lams, 1e-10), g["vd_k3/out"], 1e-11)
    close(OT.canonicalize(g["vd_k3/tensor"].copy(), lams, 1e-10), g["can_k3/out"])


@pytest.mark.parametrize("case", ["dg_cnot", "dg_zz", "dg_rand"])
def test_decompose_gate(g, case):
    h1, h2 = OT.decompose_gate(g[f"{case}/gate"], 1e-10)
    ref = lst(g, f"{case}/half")
    assert h1.shape == ref[0].shape and h2.shape == ref[1].shape
    close(h1, ref[0], 1e-10)
    close(h2, ref[1], 1e-10)


def test_apply_half_gate(g):
    h1 = lst(g, "dg_rand/half")[0]
    close(OT.apply_half_gate(g["ahg/tensor"], h1, 1), g["ahg/out"])


@pytest.mark.parametrize("case,acc,rank", [("su_acc", 1e-2, None), ("su_rank", None, 3), ("su_chi8", None, 8)])
def test_simple_update(g, case, acc, rank):
    t1, t2 = lst(g, f"{case}/t")
    h1, h2 = lst(g, f"{case}/half")
    out = OT.simple_update(t1.copy(), t2.copy(), lst(g, f"{case}/lam1"), lst(g, f"{case}/lam2"), h1, h2, 2, 0,
                           1e-10, acc, rank)
    ref = lst(g, f"{case}/out")
    for a, b in zip(out, ref):
        close(a, b, 1e-10)
