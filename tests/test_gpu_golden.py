"""The GPU path fed the reference's own recorded inputs (tests/golden).

tests/golden/*.npz hold inputs and outputs of the reference's hot-path
functions, maps, gate methods and emulators, recorded by running the
reference's source (tests/golden/make_golden.py). The CPU tests hold the
oracle to them; here the same inputs go straight through this package's CUDA
path and must give the recorded outputs:

* ``pass_through_node`` (tensor_ops.py:36-60), degrees 2-4, physical
  dimension 2 and 3, and the degree-3 node at bond 16: the generic node
  kernel (a star graph around the recorded node, BP map), the degree-3 FP64
  and FP32 kernels and the tcgen05 BF16 kernel (a 3-regular graph with the
  recorded tensor on every node);
* ``simple_update`` (tensor_ops.py:318-389) under both truncation rules and
  at bond 8 (TensorGraph.apply2_to_vidal_canonical on a graph built around
  the two recorded tensors);
* the maps (mappings/*.py) on three graphs, the TensorGraph gate methods
  (tensor_graph.py:235-446), the BP emulator with measurements
  (bp_quantum_emulator.py), the annealing loop (quantum_annealer.py:90-152)
  and the dense exact emulator (exact_quantum_emulator.py).

Tolerances: 1e-11 relative for direct FP64 outputs, 1e-10 through eigen /
singular vectors, compared gauge-invariantly where vectors enter (lambdas,
contractions of the Vidal form, two-site tensors around a bond); FP32 1e-5;
the BF16 tensor-core node update 3e-3 of the largest message entry (a CPU
model of its rounding gives 1e-3 on these inputs).
"""

import os

import numpy as np
import pytest
import torch

from dequantizer_b200 import graph as G
from dequantizer_b200 import maps as M
from dequantizer_b200.graph import Edge, MessageID, Node, TensorGraph
from tests.helpers import contract_network, rel_err, state_fidelity, to_np, two_site
from tests.test_golden_maps import GRAPHS, keyed, unpack

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-11
TOL_SVD = 1e-10


@pytest.fixture(scope="module")
def ops():
    return dict(np.load(os.path.join(HERE, "golden", "tensor_ops_golden.npz")))


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(HERE, "golden", "maps_golden.npz")))


def lst(g, key):
    return [g[f"{key}{i}"] for i in range(int(g[f"{key}_n"]))]


def close(a, b, tol):
    a, b = to_np(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    assert err <= tol, err


# ------------------------------------------------------------ node update
def star_graph(tensor):
    """A node with the recorded tensor's bonds, each to a leaf node of its
    own; bonds in the recorded order."""
    g = TensorGraph()
    c = g.add_node(tensor.shape[-1])
    leaves = [g.add_node(2) for _ in tensor.shape[:-1]]
    for leaf, dim in zip(leaves, tensor.shape[:-1]):
        g.add_edge((c, leaf), dim)
    return g, c


@pytest.mark.parametrize("case", ["ptn_k2", "ptn_k3", "ptn_k4", "ptn_k3_d3", "ptn_k3_chi16"])
def test_node_update_generic_kernel_on_recorded_inputs(ops, case):
    t = ops[f"{case}/tensor"]
    msgs, outs = lst(ops, f"{case}/msg"), lst(ops, f"{case}/out")
    g, c = star_graph(t)
    rng = np.random.default_rng(0)
    tensors = {c: t}
    messages = {}
    for e in g.get_node(c).neighbors:
        leaf = [n for n in e.neighbors if n.id != c][0]
        tensors[leaf.id] = rng.standard_normal((e.dimension, 2)) + 0j
        for key in (MessageID(leaf.id, e.id), MessageID(e.id, leaf.id), MessageID(c, e.id)):
            messages[key] = np.eye(e.dimension, dtype=complex)
    for i, e in enumerate(g.get_node(c).neighbors):
        messages[MessageID(e.id, c)] = msgs[i]
    out = M.get_belief_propagation_map(list(g.get_traversal_iterator()), True)(tensors, messages)
    for i, e in enumerate(g.get_node(c).neighbors):
        close(out[MessageID(c, e.id)], outs[i], TOL)


@pytest.mark.parametrize("precision,tol", [("fp64", TOL), ("fp32", 1e-5), ("bf16", 3e-3)])
def test_degree3_kernels_on_recorded_bond16_node(ops, precision, tol):
    """Every node of a 3-regular graph holds the recorded bond-16 tensor and
    receives the recorded messages in its bond order, so every outgoing
    message must be the recorded output of its bond."""
    from dequantizer_b200.engine import BPEngine

    t = ops["ptn_k3_chi16/tensor"]
    msgs, outs = lst(ops, "ptn_k3_chi16/msg"), lst(ops, "ptn_k3_chi16/out")
    g = G.get_random_regular_graph(16, 3, 2, 16, 9)
    eng = BPEngine(g, schedule="sync", precision=precision)
    L = eng.layout
    eng.load_tensors([t] * L.n_nodes)
    slot = (np.arange(L.n_halves) - L.node_half[L.half_node]).astype(int)
    eng.load_messages([np.eye(16, dtype=complex)] * L.n_halves, [msgs[s] for s in slot])
    eng.sweep()
    eng.check()
    got = eng.messages()
    worst = 0.0
    for h in range(L.n_halves):
        ref = outs[slot[h]]
        err = float(np.abs(to_np(got[h]).astype(np.complex128) - ref).max() / np.abs(ref).max())
        worst = max(worst, err)
    assert worst <= tol, worst
    if precision == "bf16":
        # no systematic bias: the mean signed error is far below the spread
        diff = np.stack([to_np(got[h]).astype(np.complex128) - outs[slot[h]] for h in range(L.n_halves)])
        assert abs(diff.mean()) < 0.1 * np.abs(diff).mean()


# ---------------------------------------------------------- simple update
def su_graph(t1, t2, i1, i2):
    """Two nodes joined by the bond at t1's index i1 / t2's index i2; every
    other bond goes to a leaf node of its own, in the recorded bond order."""
    g = TensorGraph()
    a = g.add_node(t1.shape[-1])
    b = g.add_node(t2.shape[-1])
    leaves_a = {k: g.add_node(2) for k in range(t1.ndim - 1) if k != i1}
    leaves_b = {k: g.add_node(2) for k in range(t2.ndim - 1) if k != i2}
    # node a's bonds in order; the shared bond is added when a reaches i1, and
    # b's bonds before i2 must already exist then, so b's leading bonds come first
    for k in range(i2):
        g.add_edge((b, leaves_b[k]), t2.shape[k])
    for k in range(t1.ndim - 1):
        if k == i1:
            g.add_edge((a, b), t1.shape[k])
        else:
            g.add_edge((a, leaves_a[k]), t1.shape[k])
    for k in range(i2 + 1, t2.ndim - 1):
        g.add_edge((b, leaves_b[k]), t2.shape[k])
    assert g.get_node(a).indices[g.find_edge(a, b).id] == i1
    assert g.get_node(b).indices[g.find_edge(a, b).id] == i2
    return g, a, b


@pytest.mark.parametrize("case,acc,rank", [("su_acc", 1e-2, None), ("su_rank", None, 3), ("su_chi8", None, 8)])
def test_simple_update_on_recorded_inputs(ops, case, acc, rank):
    t1, t2 = lst(ops, f"{case}/t")
    h1, h2 = lst(ops, f"{case}/half")
    lam1, lam2 = lst(ops, f"{case}/lam1"), lst(ops, f"{case}/lam2")
    o1, o2, lam_ref, err_ref, ent_ref = lst(ops, f"{case}/out")
    i1, i2 = 2, 0
    g, a, b = su_graph(t1, t2, i1, i2)
    gate = np.einsum("rai,rbj->abij", h1, h2)
    na, nb = g.get_node(a), g.get_node(b)
    lambdas = {}
    for node, lams in ((na, lam1), (nb, lam2)):
        for e, lam in zip(node.neighbors, lams):
            lambdas[e.id] = lam
    tensors = {a: t1, b: t2}
    _, lam_out, err, ent = g.apply2_to_vidal_canonical(a, b, tensors, lambdas, gate, 1e-10, acc, rank)
    e = g.find_edge(a, b)
    assert e.dimension == lam_ref.shape[0]
    close(lam_out[e.id], lam_ref, TOL_SVD)
    assert abs(float(err) - float(err_ref)) < 1e-10
    assert abs(float(ent) - float(ent_ref)) < 1e-10
    assert tuple(tensors[a].shape) == o1.shape and tuple(tensors[b].shape) == o2.shape
    close(two_site(tensors[a], tensors[b], i1, i2, lam_out[e.id]), two_site(o1, o2, i1, i2, lam_ref), TOL_SVD)


# ------------------------------------------------------------------- maps
@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("ordering", ["dfs", "bfs"])
@pytest.mark.parametrize("sync", [False, True])
def test_bp_sweeps_on_recorded_inputs(gold, name, ordering, sync):
    graph = GRAPHS[name]()
    tensors = keyed(graph, unpack(gold, f"{name}/tensors"))
    m = keyed(graph, unpack(gold, f"{name}/messages"))
    bp = M.get_belief_propagation_map(list(graph.get_traversal_iterator(ordering=ordering)), sync)
    for _ in range(2):
        m = bp(tensors, m)
    rec = unpack(gold, f"{name}/bp2_{ordering}_{'sync' if sync else 'async'}")
    assert set(map(repr, m)) == set(rec)
    for k, v in m.items():
        close(v, rec[repr(k)], TOL)


@pytest.mark.parametrize("name", list(GRAPHS))
def test_gauges_distances_and_densities_on_recorded_inputs(gold, name):
    graph = GRAPHS[name]()
    trav = list(graph.get_traversal_iterator())
    tensors = keyed(graph, unpack(gold, f"{name}/tensors"))
    m = keyed(graph, unpack(gold, f"{name}/messages"))
    bp = M.get_belief_propagation_map(trav)
    for _ in range(30):
        m = bp(tensors, m)
    rec30 = unpack(gold, f"{name}/messages_30")
    for k, v in m.items():
        close(v, rec30[repr(k)], TOL_SVD)
    m30 = keyed(graph, rec30)
    d = float(M.messages_frob_distance(m30, bp(tensors, m30)))
    assert abs(d - float(gold[f"{name}/frob_30_31"])) <= 1e-10 * max(1.0, abs(float(gold[f"{name}/frob_30_31"])))
    # Vidal gauge: lambdas directly, Gamma through the contraction of the Vidal form
    g_t, lam = M.get_vidal_gauge_fixing_map(trav, 1e-10)(tensors, m30)
    rec_l = {k: v.real for k, v in unpack(gold, f"{name}/vidal_lambdas").items()}
    for k, v in lam.items():
        close(v, rec_l[repr(k)], TOL_SVD)
    gv_t = keyed(graph, unpack(gold, f"{name}/vidal_tensors"))
    gv_l = keyed(graph, unpack(gold, f"{name}/vidal_lambdas"), real=True)
    if graph.nodes_number <= 12:
        psi_ref = contract_network(graph, gv_t, gv_l)
        psi_gpu = contract_network(graph, g_t, lam)
        assert 1.0 - state_fidelity(psi_ref, psi_gpu) < 1e-10
    vd = float(M.get_vidal_gauge_distance_map(trav, 1e-10)(gv_t, gv_l))
    assert abs(vd - float(gold[f"{name}/vidal_distance"])) <= 1e-10 * max(1.0, float(gold[f"{name}/vidal_distance"]))
    sym = M.get_symmetric_gauge_fixing_map(trav, 1e-10)(gv_t, gv_l)
    rec_s = unpack(gold, f"{name}/symmetric_tensors")
    for k, v in sym.items():
        close(v, rec_s[repr(k)], TOL)
    lm = M.lambdas2messages(gv_l)
    rec_m = unpack(gold, f"{name}/lambda_messages")
    for k, v in lm.items():
        close(v, rec_m[repr(k)], TOL)
    rec_rho = unpack(gold, f"{name}/density")
    for el in trav:
        if isinstance(el, Node):
            close(M.get_one_side_density_matrix(el, tensors, m30), rec_rho[repr(el.id)], TOL)


def test_graph_gate_methods_on_recorded_inputs(gold):
    """apply1, apply2_to_vidal_canonical (rank cap, accuracy cap, none),
    truncate and apply2 on the 2x3x2 lattice's recorded Vidal form, as the
    reference ran them: lambdas, truncation errors, entropies and bond
    dimensions directly, tensors through the contracted state (Gamma is
    fixed up to singular-vector phases)."""
    graph = GRAPHS["lat232"]()
    edges = [el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, Edge)]
    tensors = {k: torch.from_numpy(v).cuda() for k, v in keyed(graph, unpack(gold, "lat232/vidal_tensors")).items()}
    lambdas = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
               for k, v in keyed(graph, unpack(gold, "lat232/vidal_lambdas"), real=True).items()}
    rx = np.array([[np.cos(0.3), -1j * np.sin(0.3)], [-1j * np.sin(0.3), np.cos(0.3)]])
    cnot = np.eye(4, dtype=complex)[[0, 1, 3, 2]].reshape(2, 2, 2, 2)
    zz = np.diag(np.exp(1j * np.array([0.3, -0.3, -0.3, 0.3]))).reshape(2, 2, 2, 2)
    rnd = gold["ops/gate_rnd"]
    first = next(el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, Node))
    graph.apply1(first.id, tensors, rx)
    rec = keyed(graph, unpack(gold, "lat232/ops/after_apply1"))
    for k, v in tensors.items():
        close(v, rec[k], TOL)

    def state(ts, ls):
        return contract_network(graph, ts, ls)

    steps = [(cnot, edges[0], None, 3), (rnd, edges[1], 1e-3, None), (zz, edges[2], None, None)]
    for i, (gate, edge, acc, rank) in enumerate(steps):
        a, b = edge.id
        _, _, err, ent = graph.apply2_to_vidal_canonical(a, b, tensors, lambdas, gate, 1e-10, acc, rank)
        assert [e.dimension for e in edges] == list(gold[f"ops/step{i}_edge_dims"])
        rec_t = keyed(graph, unpack(gold, f"lat232/ops/step{i}_tensors"))
        rec_l = keyed(graph, unpack(gold, f"lat232/ops/step{i}_lambdas"), real=True)
        for k, v in lambdas.items():
            close(v, rec_l[k], TOL_SVD)
        assert abs(float(err) - float(gold[f"ops/step{i}_err"])) < 1e-8
        assert abs(float(ent) - float(gold[f"ops/step{i}_entropy"])) < 1e-10
        assert 1.0 - state_fidelity(state(tensors, lambdas), state(rec_t, rec_l)) < 1e-10
    tensors, lambdas = graph.truncate(tensors, lambdas, 1e-2)
    assert [e.dimension for e in edges] == list(gold["ops/truncated_edge_dims"])
    rec_t = keyed(graph, unpack(gold, "lat232/ops/truncated_tensors"))
    rec_l = keyed(graph, unpack(gold, "lat232/ops/truncated_lambdas"), real=True)
    for k, v in lambdas.items():
        close(v, rec_l[k], TOL_SVD)
    psi_t = state(tensors, lambdas)
    assert 1.0 - state_fidelity(psi_t, state(rec_t, rec_l)) < 1e-10
    a, b = edges[3].id
    graph.apply2(a, b, tensors, rnd, 1e-10)
    assert [e.dimension for e in edges] == list(gold["ops/apply2_edge_dims"])
    rec_t = keyed(graph, unpack(gold, "lat232/ops/apply2_tensors"))
    # apply2 grows a bond without lambdas: compare the contraction of the
    # tensors alone (Gamma's singular-vector phases are diagonal unitaries on
    # the bonds and cancel in it)
    assert 1.0 - state_fidelity(state(tensors, None), state(rec_t, None)) < 1e-10


def test_truncate_matches_oracle_on_its_own():
    """TensorGraph.truncate (tensor_graph.py:235-258) on the GPU against the
    oracle from the same Vidal form, under the accuracy rule and the rank cap:
    identical tensors (a slice, no arithmetic), lambdas and bond dimensions."""
    from oracle import maps as OM
    from tests.helpers import random_messages, random_tensors

    for acc, rank in ((1e-2, None), (None, 3), (1e-6, 2)):
        g_ref = G.get_random_regular_graph(8, 3, 2, 6, 4)
        g_gpu = G.get_random_regular_graph(8, 3, 2, 6, 4)
        tensors = random_tensors(g_ref, 3)
        trav = list(g_ref.get_traversal_iterator())
        msgs = random_messages(g_ref, 4)
        bp = OM.get_belief_propagation_map(trav)
        for _ in range(40):
            msgs = bp(tensors, msgs)
        r_t, r_l = OM.get_vidal_gauge_fixing_map(trav, 1e-10)(tensors, msgs)
        g_t = {k: torch.from_numpy(v).cuda() for k, v in r_t.items()}
        g_l = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in r_l.items()}
        r_t, r_l = OM.truncate(g_ref, dict(r_t), dict(r_l), acc, rank)
        g_t, g_l = g_gpu.truncate(g_t, g_l, acc, rank)
        for eid in g_ref.edges:
            assert g_gpu.get_edge(eid).dimension == g_ref.get_edge(eid).dimension
            assert torch.equal(g_l[eid].cpu(), torch.from_numpy(np.ascontiguousarray(r_l[eid])))
        for nid in g_ref.nodes:
            assert g_gpu.get_node(nid).bond_shape == g_ref.get_node(nid).bond_shape
            assert tuple(g_t[nid].shape) == r_t[nid].shape
            assert np.array_equal(to_np(g_t[nid]), r_t[nid])


# ------------------------------------------------------------ emulators
def test_bp_emulator_on_recorded_run(gold):
    """The GPU BPQuantumEmulator replays the reference's recorded run on the
    infinite heavy-hex cell (key 42, bond <= 4, a regauge per layer, three
    kicked-Ising layers, then two measurements): densities after each layer
    and after the measurements, outcomes, truncation errors, entropies and
    Vidal distances."""
    from dequantizer_b200.emulator import BPQuantumEmulator

    lat = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    trav = list(lat.get_traversal_iterator())
    em = BPQuantumEmulator(lat, 42, 4, lat.edges_number, 1e-7, 100)
    rzz = np.diag(np.exp(np.array([1j, -1j, -1j, 1j]) * np.pi / 4)).reshape(2, 2, 2, 2)
    rx = np.array([[np.cos(0.4), -1j * np.sin(0.4)], [-1j * np.sin(0.4), np.cos(0.4)]])
    nodes = [el.id for el in trav if isinstance(el, Node)]
    for layer in range(3):
        for n in nodes:
            em.apply_q1(rx, n)
        for el in trav:
            if isinstance(el, Edge):
                em.apply_q2(rzz, *el.id)
        close(torch.stack([em.dens_q1(n) for n in nodes]), gold[f"emu/rho_{layer}"], 1e-9)
    outcomes = []
    for i in gold["emu/measured"]:
        sample = np.random.default_rng(int(em._rng.integers(0, 2**31 - 1))).uniform(size=(1,))[0]
        outcomes.append(em.measure(nodes[int(i)], sample))
    assert outcomes == list(gold["emu/outcomes"])
    # after a measurement the state is re-canonicalised from fresh messages
    # down to the BP accuracy (1e-7): rounding can move the stopping sweep, so
    # densities agree to that accuracy
    close(torch.stack([em.dens_q1(n) for n in nodes]), gold["emu/rho_after_measure"], 1e-7)
    errs = np.array([float(x) for x in em.truncation_errors])
    assert errs.shape == gold["emu/truncation_errors"].shape
    assert np.abs(errs - gold["emu/truncation_errors"]).max() < 1e-9
    ents = np.array([float(x) for x in em.entropies])
    assert np.abs(ents - gold["emu/entropies"]).max() < 1e-9
    # distances after the layers agree closely; the two re-canonicalisations
    # after the measurements stop at the BP accuracy (1e-7) from fresh
    # messages, where rounding moves the stopping point
    after, after_ref = to_np(em.after_regauging_vidal_distances), gold["emu/after_regauging"]
    n_meas = len(gold["emu/measured"])
    assert after.shape == after_ref.shape
    assert np.abs(after[:-n_meas] - after_ref[:-n_meas]).max() < 1e-9
    assert np.all(after[-n_meas:] <= 1e-7) and np.all(after_ref[-n_meas:] <= 1e-7)
    assert np.abs(to_np(em.truncated_affected_vidal_distances) - gold["emu/truncated_affected"]).max() < 1e-9


def test_annealer_on_recorded_run(gold):
    """The GPU annealing loop (first-order steps, the reference's scheduler)
    replays the reference's run_quantum_annealer on its recorded 10-spin
    instance (key 7, bond <= 4, six steps of 0.2)."""
    from dequantizer_b200 import workloads as W

    energy = W.EnergyFunction(gold["anneal/amps"], gold["anneal/pairs"], gold["anneal/fields"])
    res = W.run_quantum_annealer(energy, W.scheduler(0.2, lambda t: 1 - t, 6), key=7, max_chi=4,
                                 gates_number_per_regauging=len(energy.coupled_spin_pairs), accuracy=1e-7,
                                 max_belief_propagation_iterations=100)
    close(res.density_matrices, gold["anneal/rho"], 1e-9)
    assert np.abs(res.truncation_errors - gold["anneal/truncation_errors"]).max() < 1e-9
    assert np.abs(res.entropies - gold["anneal/entropies"]).max() < 1e-9
    ref_vd = gold["anneal/after_regauging"]
    assert len(res.vidal_distances_after_regauging) == len(ref_vd)
    assert np.abs(res.vidal_distances_after_regauging - ref_vd).max() < 1e-9


def test_dense_emulator_on_recorded_run(gold):
    """The GPU dense state-vector emulator replays the reference's
    ExactQuantumEmulator run on the 2x3 lattice."""
    from dequantizer_b200.dense import DenseStateEmulator

    lat = G.get_nd_lattice([2, 3], 2, 2, True)
    trav = list(lat.get_traversal_iterator())
    nodes = [el.id for el in trav if isinstance(el, Node)]
    edges = [el.id for el in trav if isinstance(el, Edge)]
    em = DenseStateEmulator(lat)
    em.set_to_product_state({n: int(b) for n, b in zip(nodes, gold["exact/bits"])})
    for layer in range(2):
        for n, g in zip(nodes, gold[f"exact/g1_{layer}"]):
            em.apply_q1(g, n)
        for e, g in zip(edges, gold[f"exact/g2_{layer}"]):
            em.apply_q2(g, e[0], e[1])
        close(torch.stack([em.dens_q1(n) for n in nodes]), gold[f"exact/rho_{layer}"], 1e-12)
    stream = np.random.default_rng(5)
    outcomes = []
    for i in gold["exact/measured"]:
        sample = np.random.default_rng(int(stream.integers(0, 2**31 - 1))).uniform(size=(1,))[0]
        stream.integers(0, 2**31 - 1)
        outcomes.append(em.measure(nodes[int(i)], sample))
    assert outcomes == list(gold["exact/outcomes"])
    close(torch.stack([em.dens_q1(n) for n in nodes]), gold["exact/rho_after"], 1e-12)
