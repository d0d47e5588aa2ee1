"""dqz_simple_update_noalloc against dqz_simple_update.

The no-allocation entry point serves callers that cannot allocate device
memory themselves (a host program that passes only its own input and output
buffers, or a loop that cannot pay for cudaMalloc's synchronisation). It
must give the same Gamma tensors, lambdas, truncation errors and entropies
as the allocating entry point, also when it is called twice in a row and the
library-owned scratch array still holds the previous call's data.

The test allocates its inputs and outputs with torch (the caller's job); the
entry point itself takes no scratch argument. This file is named so pytest
collects it last.
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import _lib
from dequantizer_b200.gates import decompose_gates
from dequantizer_b200.graph import get_random_regular_graph
from dequantizer_b200.layout import GraphLayout
from dequantizer_b200.tensor_graph_ops import simple_update_shapes

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _state(seed):
    g = get_random_regular_graph(12, 3, 2, 4, seed)
    nodes, edges = list(g.nodes.values()), list(g.edges.values())
    max_chi = 6
    # room for every bond to grow to max_chi
    cap = [2 * max_chi**3 for _ in nodes]
    L = GraphLayout(nodes, edges, [4] * len(edges), node_capacity=cap, edge_capacity=[max_chi] * len(edges))
    rng = np.random.default_rng(seed)
    T = L.new_tensor_arena()
    for v in range(L.n_nodes):
        size = 2 * 4**3
        z = rng.standard_normal((size, 2))
        T[int(L.node_off[v]) : int(L.node_off[v]) + size] = torch.from_numpy(z[:, 0] + 1j * z[:, 1])
    lam = L.new_lam_arena()
    for e in range(L.n_edges):
        lam[int(L.edge_lam_off[e]) : int(L.edge_lam_off[e]) + 4] = torch.from_numpy(
            np.sort(rng.uniform(0.05, 1.0, 4))[::-1].copy())
    return g, L, T, lam, max_chi, rng


def _batch(L, used_edges, rng, max_chi):
    """A node-disjoint set of edges with random two-site gates."""
    taken, jobs = set(), []
    for e in range(L.n_edges):
        if e in used_edges:
            continue
        h0, h1 = L.edge_half[2 * e], L.edge_half[2 * e + 1]
        a, b = int(L.half_node[h0]), int(L.half_node[h1])
        if a in taken or b in taken:
            continue
        taken |= {a, b}
        jobs.append(e)
    n = len(jobs)
    z = rng.standard_normal((n, 4, 4, 2))
    q, _ = np.linalg.qr(z[..., 0] + 1j * z[..., 1])
    flat, ranks, _ = decompose_gates(q.reshape(n, 2, 2, 2, 2), 1e-10)
    rows, cols = 1, 1
    for j, e in enumerate(jobs):
        h0, h1 = L.edge_half[2 * e], L.edge_half[2 * e + 1]
        a, b = int(L.half_node[h0]), int(L.half_node[h1])
        i0, i1 = int(h0 - L.node_half[a]), int(h1 - L.node_half[b])
        m1, m2, k, new, _ = simple_update_shapes(L.node_dims(a), 2, i0, L.node_dims(b), 2, i1, int(ranks[j]), max_chi)
        rows, cols = max(rows, m1, m2), max(cols, k)
        L.edge_chi[e] = new
    return jobs, flat, ranks, rows, cols


def _run(entry, L, T, lam, jobs, flat, ranks, rows, cols, max_chi):
    dev = T.device
    n = len(jobs)
    edges = torch.tensor(jobs, dtype=torch.int32, device=dev)
    first = torch.ones(n, dtype=torch.uint8, device=dev)
    halves = torch.from_numpy(flat.reshape(n, -1)).to(dev)
    rk = torch.from_numpy(ranks).to(dev)
    err = torch.empty(n, dtype=torch.float64, device=dev)
    ent = torch.empty(n, dtype=torch.float64, device=dev)
    args = [L.gptr, T.data_ptr(), lam.data_ptr(), edges.data_ptr(), first.data_ptr(), halves.data_ptr(), rk.data_ptr(),
            n, 1e-10, max_chi, rows, cols, err.data_ptr(), ent.data_ptr()]
    if entry == "dqz_simple_update":
        scratch = torch.empty(_lib.lib().dqz_simple_update_scratch_bytes(n, rows, cols), dtype=torch.uint8,
                              device=dev)
        args.append(scratch.data_ptr())
    args.append(_lib.stream_handle())
    _lib.call(entry, *args)
    torch.cuda.synchronize()
    return err, ent


@pytest.mark.parametrize("stride_rows", [None, 12000, 30000])
def test_noalloc_matches_allocating_entry_point_twice(stride_rows):
    """stride_rows: a larger row bound than the jobs need (the kernels use it
    only as the stride of their scratch slices), so that 2 or 1 job slices
    fit in the library's array and the jobs of one call share them in turn."""
    g, L_a, T_a, lam_a, max_chi, rng = _state(3)
    _, L_b, T_b, lam_b, _, _ = _state(3)
    rng_a, rng_b = np.random.default_rng(99), np.random.default_rng(99)
    used_a, used_b = set(), set()
    for call in range(2):
        jobs, flat, ranks, rows, cols = _batch(L_a, used_a, rng_a, max_chi)
        jobs_b, flat_b, ranks_b, rows_b, cols_b = _batch(L_b, used_b, rng_b, max_chi)
        assert jobs == jobs_b and rows == rows_b and cols == cols_b
        if stride_rows is not None:
            cols = 16
            rows = rows_b = stride_rows
            slots = (32 << 20) // (64 * rows * cols)
            assert slots in (1, 2) and len(jobs) > slots
        used_a |= set(jobs)
        used_b |= set(jobs)
        err_a, ent_a = _run("dqz_simple_update", L_a, T_a, lam_a, jobs, flat, ranks, rows, cols, max_chi)
        err_b, ent_b = _run("dqz_simple_update_noalloc", L_b, T_b, lam_b, jobs, flat_b, ranks_b, rows, cols,
                            max_chi)
        assert torch.equal(L_a.d_edge_chi, L_b.d_edge_chi)
        scale = float(T_a.abs().max())
        assert float((T_a - T_b).abs().max()) <= TOL * scale, call
        assert float((lam_a - lam_b).abs().max()) <= TOL * float(lam_a.abs().max()), call
        assert float((err_a - err_b).abs().max()) <= TOL, call
        assert float((ent_a - ent_b).abs().max()) <= TOL, call


def test_noalloc_rejects_jobs_larger_than_its_array():
    g, L, T, lam, max_chi, rng = _state(5)
    dev = T.device
    one_i = torch.zeros(1, dtype=torch.int32, device=dev)
    one_u = torch.ones(1, dtype=torch.uint8, device=dev)
    halves = torch.zeros(2 * 4 * _lib.MAX_PHYS**2, dtype=torch.complex128, device=dev)
    out = torch.empty(1, dtype=torch.float64, device=dev)
    rows = (32 << 20) // (64 * 64) + 1  # one job would need more than 32 MiB
    status = _lib.lib().dqz_simple_update_noalloc(L.gptr, T.data_ptr(), lam.data_ptr(), one_i.data_ptr(),
                                                  one_u.data_ptr(), halves.data_ptr(), one_i.data_ptr(), 1, 1e-10,
                                                  4, rows, 64, out.data_ptr(), out.data_ptr(),
                                                  _lib.stream_handle())
    assert status == _lib.DQZ_ERR_UNSUPPORTED
