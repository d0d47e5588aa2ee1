"""GPU parity against the FP64 oracle at the shapes the workloads run.

* The simple update (tensor_ops.py:265-389) between degree-3 nodes at bond 16
  (a 512 x 32 matrix per side for a rank-2 gate, 512 x 64 for a rank-4 one:
  the batched-annealing and gradient workloads) and at bond 32 (2048 x 64,
  truncated back to 32: the 127-qubit kicked-Ising workload), under the
  rank-cap rule and the accuracy rule.
* The generic node update and the one-CTA gauge kernels at bond 32 on the
  heavy-hex cell, whose nodes have degree 2 and 3 (tensor_ops.py:36-60,
  108-175; the kicked-Ising regauges).
* The batched annealer against per-instance oracle emulator runs at bond
  caps 8 and 16, with the bonds reaching the cap
  (quantum_annealer.py:90-152, bp_quantum_emulator.py:144-300).

Tolerances as elsewhere: lambdas, truncation errors and entropies 1e-10,
two-site tensors around the updated bond (gauge-invariant) 1e-10 relative,
densities 1e-9.
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import graph as G
from dequantizer_b200 import maps as M
from dequantizer_b200 import workloads as W
from dequantizer_b200.graph import Node
from oracle import maps as OM
from oracle.emulator import BPQuantumEmulator as OracleEmulator
from tests.helpers import random_messages, random_tensors, rel_err, to_np, two_site

pytestmark = pytest.mark.gpu

TOL_SVD = 1e-10


def vidal_like_lambdas(graph, rng):
    """Descending positive spectra spread over three decades, unit norm."""
    out = {}
    for eid, e in graph.edges.items():
        lam = np.sort(10.0 ** rng.uniform(-3, 0, e.dimension))[::-1]
        out[eid] = lam / np.linalg.norm(lam)
    return out


def zz_gate(rng):
    return np.diag(np.exp(1j * rng.uniform(-np.pi, np.pi, 4))).reshape(2, 2, 2, 2)


def unitary_gate(rng):
    z = rng.standard_normal((4, 4, 2))
    q, _ = np.linalg.qr(z[..., 0] + 1j * z[..., 1])
    return q.reshape(2, 2, 2, 2)


@pytest.mark.parametrize("chi,kind,accuracy,max_rank", [
    (16, "zz", None, 16),      # 512 x 32 per side, cut 32 -> 16
    (16, "zz", 1e-3, None),    # accuracy rule
    (16, "unitary", None, 16),  # rank-4 gate: 512 x 64, cut 64 -> 16
    (32, "zz", None, 32),      # 2048 x 64 per side, cut 64 -> 32
    (32, "zz", 1e-4, 48),      # both rules
])
def test_simple_update_at_production_shapes(chi, kind, accuracy, max_rank):
    rng = np.random.default_rng(chi + (1 if kind == "unitary" else 0) + (2 if accuracy else 0))
    g_ref = G.get_random_regular_graph(8, 3, 2, chi, 5)
    g_gpu = G.get_random_regular_graph(8, 3, 2, chi, 5)
    tensors = random_tensors(g_ref, chi)
    lambdas = vidal_like_lambdas(g_ref, rng)
    r_t, r_l = dict(tensors), dict(lambdas)
    g_t = {k: torch.from_numpy(v).cuda() for k, v in tensors.items()}
    g_l = {k: torch.from_numpy(v.copy()).cuda() for k, v in lambdas.items()}
    edges = list(g_ref.edges)
    for a, b in (edges[0], edges[4]):
        gate = zz_gate(rng) if kind == "zz" else unitary_gate(rng)
        _, _, er, en = OM.apply2_to_vidal_canonical(g_ref, a, b, r_t, r_l, gate, 1e-10, accuracy, max_rank)
        _, _, eg, ng = g_gpu.apply2_to_vidal_canonical(a, b, g_t, g_l, gate, 1e-10, accuracy, max_rank)
        edge = g_ref.find_edge(a, b)
        assert g_gpu.find_edge(a, b).dimension == edge.dimension
        assert tuple(g_t[a].shape) == r_t[a].shape and tuple(g_t[b].shape) == r_t[b].shape
        assert rel_err(g_l[edge.id], r_l[edge.id]) < TOL_SVD
        assert abs(float(eg) - er) < 1e-10
        assert abs(float(ng) - en) < 1e-10
        n1, n2 = g_ref.get_node(a), g_ref.get_node(b)
        i1, i2 = n1.indices[edge.id], n2.indices[edge.id]
        assert rel_err(two_site(g_t[a], g_t[b], i1, i2, g_l[edge.id]),
                       two_site(r_t[a], r_t[b], i1, i2, r_l[edge.id])) < TOL_SVD
        # the next gate starts from identical inputs on both sides
        g_t[a], g_t[b] = torch.from_numpy(r_t[a]).cuda(), torch.from_numpy(r_t[b]).cuda()
        g_l[edge.id] = torch.from_numpy(r_l[edge.id].copy()).cuda()


@pytest.mark.parametrize("path", ["onchip", "global_scratch"])
@pytest.mark.parametrize("max_rank", [None, 12])
def test_simple_update_on_uneven_shapes(path, max_rank):
    """Degree-2 and degree-3 nodes with uneven bonds (the heavy-hex cell with
    bonds of 2, 8 and 16): jobs whose matrices have 256 rows or more on one
    side only, wide and tall factors, with and without a rank cap, through the
    on-chip form (default) and through the global-scratch kernel (knob
    su_onchip = 1), each against the oracle."""
    from dequantizer_b200 import autotune

    rng = np.random.default_rng(7 if max_rank else 8)
    g_ref = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    g_gpu = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    dims = {eid: int(rng.choice([2, 8, 16])) for eid in g_ref.edges}
    for gg in (g_ref, g_gpu):
        for eid, e in gg.edges.items():
            e.dimension = dims[eid]
        gg.refresh_bond_shapes()
    tensors = random_tensors(g_ref, 41)
    lambdas = vidal_like_lambdas(g_ref, rng)
    r_t, r_l = dict(tensors), dict(lambdas)
    g_t = {k: torch.from_numpy(v).cuda() for k, v in tensors.items()}
    g_l = {k: torch.from_numpy(v.copy()).cuda() for k, v in lambdas.items()}
    autotune.set_knobs({"su_onchip": 1 if path == "global_scratch" else 0})
    try:
        for a, b in list(g_ref.edges)[:8]:
            gate = zz_gate(rng) if rng.uniform() < 0.5 else unitary_gate(rng)
            edge = g_ref.find_edge(a, b)
            n1, n2 = g_ref.get_node(a), g_ref.get_node(b)
            if edge.dimension * 4 > 64:
                gate = zz_gate(rng)  # bond x gate rank stays within the kernels' 64 columns
            _, _, er, en = OM.apply2_to_vidal_canonical(g_ref, a, b, r_t, r_l, gate, 1e-10, None, max_rank)
            _, _, eg, ng = g_gpu.apply2_to_vidal_canonical(a, b, g_t, g_l, gate, 1e-10, None, max_rank)
            assert g_gpu.find_edge(a, b).dimension == edge.dimension
            assert tuple(g_t[a].shape) == r_t[a].shape and tuple(g_t[b].shape) == r_t[b].shape
            assert rel_err(g_l[edge.id], r_l[edge.id]) < TOL_SVD
            assert abs(float(eg) - er) < 1e-10 and abs(float(ng) - en) < 1e-10
            i1, i2 = n1.indices[edge.id], n2.indices[edge.id]
            assert rel_err(two_site(g_t[a], g_t[b], i1, i2, g_l[edge.id]),
                           two_site(r_t[a], r_t[b], i1, i2, r_l[edge.id])) < TOL_SVD
            g_t[a], g_t[b] = torch.from_numpy(r_t[a]).cuda(), torch.from_numpy(r_t[b]).cuda()
            g_l[edge.id] = torch.from_numpy(r_l[edge.id].copy()).cuda()
    finally:
        autotune.set_knobs({"su_onchip": 0})


def heavy_hex_cell_at(chi):
    g = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    for e in g.edges.values():
        e.dimension = chi
    g.refresh_bond_shapes()
    return g


@pytest.mark.parametrize("sync", [True, False])
def test_generic_node_update_at_bond32_on_heavy_hex(sync):
    g = heavy_hex_cell_at(32)
    assert {n.degree for n in g.nodes.values()} == {2, 3}
    trav = list(g.get_traversal_iterator(ordering="dfs"))
    tensors = random_tensors(g, 31)
    messages = random_messages(g, 32)
    ref = OM.get_belief_propagation_map(trav, sync)
    gpu = M.get_belief_propagation_map(trav, sync)
    r, q = messages, messages
    for _ in range(2):
        r = ref(tensors, r)
        q = gpu(tensors, q)
    for k in r:
        assert rel_err(q[k], r[k]) < 1e-11, k


def test_vidal_gauge_and_distance_at_bond32_on_heavy_hex():
    """Bonds above 16 take the one-CTA-per-edge gauge kernels."""
    g = heavy_hex_cell_at(32)
    trav = list(g.get_traversal_iterator())
    tensors = random_tensors(g, 33)
    bp = OM.get_belief_propagation_map(trav)
    msgs = random_messages(g, 34)
    for _ in range(60):
        new = bp(tensors, msgs)
        d = OM.messages_frob_distance(new, msgs)
        msgs = new
        if d < 1e-12:
            break
    eps = 1e-10
    r_t, r_l = OM.get_vidal_gauge_fixing_map(trav, eps)(tensors, msgs)
    g_t, g_l = M.get_vidal_gauge_fixing_map(trav, eps)(tensors, msgs)
    for eid in r_l:
        assert rel_err(g_l[eid], r_l[eid]) < TOL_SVD
    vd = OM.get_vidal_gauge_distance_map(trav, eps)
    vd_gpu_gauge = vd({k: to_np(v) for k, v in g_t.items()}, {k: to_np(v) for k, v in g_l.items()})
    assert abs(vd_gpu_gauge - vd(r_t, r_l)) < 1e-9
    vd_by_gpu = float(M.get_vidal_gauge_distance_map(trav, eps)(r_t, r_l))
    assert abs(vd_by_gpu - vd(r_t, r_l)) < 1e-10 * max(1.0, vd(r_t, r_l))


def oracle_annealing(energy, steps, max_chi, accuracy, second_order):
    """The reference annealing loop on the oracle emulator (synchronous BP,
    key 1: the batched annealer's message seeds)."""
    g = W.tensor_graph_of(energy)
    em = OracleEmulator(g, 1, max_chi, energy.edges_number, accuracy, 100, synchronous_update=True)
    n = g.nodes_number
    deg = {nid: g.get_node(nid).degree for nid in g.nodes}
    for nid in range(n):
        em.apply_q1(W.HADAMARD, nid)
    for mix, coup in steps:
        if second_order:
            for nid in range(n):
                em.apply_q1(W.q1_gate(mix / 2), nid)
        for (a, b), J in zip(energy.coupled_spin_pairs, energy.coupling_amplitudes):
            a, b = int(a), int(b)
            em.apply_q2(W.q2_gate(J, energy.fields[a] / deg[a], energy.fields[b] / deg[b], coup), a, b)
        for nid in range(n):
            em.apply_q1(W.q1_gate(mix / 2 if second_order else mix), nid)
    rho = np.stack([em.dens_q1(i) for i in range(n)])
    bonds = [e.dimension for e in g.edges.values()]
    return rho, np.array(em.truncation_errors), bonds


@pytest.mark.parametrize("max_chi,sizes", [(8, (10, 12, 14)), (16, (16, 20))])
def test_batched_annealer_matches_oracle_per_instance(max_chi, sizes):
    """Instances of uneven size advanced together at bond caps 8 and 16
    (second-order steps, the bench's form) against each instance run alone
    through the oracle emulator: densities 1e-9, truncation errors 1e-9, and
    the bond cap reached with truncation."""
    from dequantizer_b200.annealing import BatchedAnnealer

    energies = [W.random_regular_energy(n, 3, seed=40 + n, field_std=0.5) for n in sizes]
    steps = list(W.scheduler(0.5, lambda t: 1 - t, 8))
    ba = BatchedAnnealer(energies, max_chi=max_chi, accuracy=1e-8, max_belief_propagation_iterations=100)
    rho_b = ba.run(steps, second_order=True)
    errs_b = ba.truncation_errors()
    reached, truncated = 0, 0.0
    for k, en in enumerate(energies):
        rho, errs, bonds = oracle_annealing(en, steps, max_chi, 1e-8, True)
        assert np.abs(rho_b[k] - rho).max() < 1e-9
        assert np.abs(errs_b[k] - errs).max() < 1e-9
        reached, truncated = max(reached, max(bonds)), max(truncated, float(errs.max()))
    assert reached == max_chi and truncated > 1e-6


@pytest.mark.parametrize("chi,nn", [(16, 600), (32, 96)])
def test_simple_update_forms_agree_on_a_batch(chi, nn):
    """One dqz_simple_update batch of node-disjoint bond-16 jobs (more jobs
    than SMs) and of bond-32 jobs (2048 x 64 per side, above shared memory)
    through each form the knob selects: the one-CTA global-scratch kernel
    (su_onchip = 1), the cluster forms at any batch size (2), the default rule
    (0), the default without the global-workspace cluster form (3) and the
    global-workspace cluster form with 256 threads for every job (4). Lambdas,
    truncation errors and entropies agree to 1e-12, and the two-site tensors
    around the updated bonds (gauge-invariant) to 1e-10 relative."""
    from dequantizer_b200 import _lib, autotune
    from dequantizer_b200.gates import decompose_gates
    from dequantizer_b200.layout import GraphLayout

    g = G.get_random_regular_graph(nn, 3, 2, chi, 1)
    nodes, edges = list(g.nodes.values()), list(g.edges.values())
    L = GraphLayout(nodes, edges, [chi] * len(edges))
    rng = np.random.default_rng(chi)
    T0 = L.new_tensor_arena()
    z = rng.standard_normal((T0.numel(), 2))
    T0.copy_(torch.from_numpy(z[:, 0] + 1j * z[:, 1]))
    lam0 = L.new_lam_arena()
    lam0.copy_(torch.from_numpy(np.concatenate([np.sort(10 ** rng.uniform(-3, 0, chi))[::-1]
                                                for _ in range(L.n_edges)])))
    taken, jobs = set(), []
    for e in range(L.n_edges):
        a, b = int(L.half_node[L.edge_half[2 * e]]), int(L.half_node[L.edge_half[2 * e + 1]])
        if a not in taken and b not in taken:
            taken |= {a, b}
            jobs.append(e)
    n = len(jobs)
    gates = np.zeros((n, 4, 4), complex)
    gates[:, range(4), range(4)] = np.exp(1j * rng.uniform(-3, 3, (n, 4)))
    flat, ranks, _ = decompose_gates(gates.reshape(n, 2, 2, 2, 2), 1e-10)
    rows, cols = 2 * chi * chi, chi * int(ranks.max())
    dev = torch.device("cuda", 0)
    ed = torch.tensor(jobs, dtype=torch.int32, device=dev)
    first = torch.ones(n, dtype=torch.uint8, device=dev)
    halves = torch.from_numpy(flat.reshape(n, -1)).to(dev)
    rk = torch.from_numpy(ranks).to(dev)
    out = {}
    try:
        for knob in (1, 2, 0, 3, 4):
            autotune.set_knobs({"su_onchip": knob})
            T, lam = T0.clone(), lam0.clone()
            err = torch.empty(n, dtype=torch.float64, device=dev)
            ent = torch.empty_like(err)
            scratch = torch.empty(_lib.lib().dqz_simple_update_scratch_bytes(n, rows, cols), dtype=torch.uint8,
                                  device=dev)
            _lib.call("dqz_simple_update", L.gptr, T.data_ptr(), lam.data_ptr(), ed.data_ptr(), first.data_ptr(),
                      halves.data_ptr(), rk.data_ptr(), n, 1e-10, chi, rows, cols, err.data_ptr(), ent.data_ptr(),
                      scratch.data_ptr(), _lib.stream_handle())
            torch.cuda.synchronize()
            L.edge_chi[:] = chi  # max_rank = chi keeps every bond at chi
            L.push_edge_chi()
            out[knob] = (T, lam, err, ent)
    finally:
        autotune.set_knobs({"su_onchip": 0})
    ref = out[1]
    for knob in (2, 0, 3, 4):
        T, lam, err, ent = out[knob]
        assert float((lam - ref[1]).abs().max()) < 1e-12
        assert float((err - ref[2]).abs().max()) < 1e-12
        assert float((ent - ref[3]).abs().max()) < 1e-12
        ta, tr = L.unpack_tensors(T), L.unpack_tensors(ref[0])
        for e in jobs[:: max(1, n // 8)]:
            ha, hb = int(L.edge_half[2 * e]), int(L.edge_half[2 * e + 1])
            a, b = int(L.half_node[ha]), int(L.half_node[hb])
            ia, ib = ha - int(L.node_half[a]), hb - int(L.node_half[b])
            got = two_site(ta[a], ta[b], ia, ib, L.lambda_view(lam, e))
            want = two_site(tr[a], tr[b], ia, ib, L.lambda_view(ref[1], e))
            assert rel_err(got, want) < 1e-10
