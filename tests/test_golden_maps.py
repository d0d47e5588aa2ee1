"""The oracle's maps against the reference's own maps on deterministic graphs.

tests/golden/maps_golden.npz (tests/golden/make_golden.py) holds, for a
2x3x2 lattice (bond 2), a 2x2x2 lattice (bond 3) and the infinite heavy-hex
cell, what the reference's dequantizer/src/mappings produce:
* the DFS and BFS traversal orders;
* two BP sweeps in each schedule (asynchronous / synchronous, DFS / BFS order)
  from seeded tensors and messages;
* after 30 asynchronous sweeps: the message distance to the next sweep, the
  Vidal gauge (tensors and lambdas), the Vidal distance, the symmetric gauge,
  lambdas2messages and every node's one-site density matrix.
Graphs come from this package's own constructors, so the traversal check
also pins the graph structure. Each oracle map gets the reference's inputs
and must give its outputs (1e-12; 1e-10 after 30 sweeps and where
eigen / singular vectors enter).
"""

import os

import numpy as np
import pytest

from dequantizer_b200 import graph as G
from dequantizer_b200.graph import Node
from oracle import maps as OM

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "maps_golden.npz")
GRAPHS = {
    "lat232": lambda: G.get_nd_lattice([2, 3, 2], 2, 2, True),
    "lat222_chi3": lambda: G.get_nd_lattice([2, 2, 2], 2, 3, True),
    "hexinf": G.get_heavy_hex_ibm_eagle_lattice_infinite,
}


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLDEN))


def unpack(gold, prefix):
    """repr(key) -> array of one recorded dict."""
    keys = gold[f"{prefix}/keys"]
    ndim, dims, data = gold[f"{prefix}/ndim"], gold[f"{prefix}/dims"], gold[f"{prefix}/data"]
    out, d0, v0 = {}, 0, 0
    for k, nd in zip(keys, ndim):
        shape = tuple(int(x) for x in dims[d0:d0 + nd])
        n = int(np.prod(shape)) if shape else 1
        out[str(k)] = data[v0:v0 + n].reshape(shape)
        d0, v0 = d0 + nd, v0 + n
    return out


def keyed(graph, recorded, real=False):
    """A recorded dict re-keyed by this package's IDs (elements and messages)."""
    ids = {}
    for el in graph.get_traversal_iterator():
        ids[repr(el.id)] = el.id
    for k in graph.init_messages(lambda md: None):
        ids[repr(k)] = k
    return {ids[k]: (v.real if real else v) for k, v in recorded.items()}


def close(a, b, tol):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)


def close_dicts(a, recorded, tol):
    """``a`` keyed by IDs, ``recorded`` by their repr."""
    assert set(map(repr, a)) == set(recorded)
    for k, v in a.items():
        close(v, recorded[repr(k)], tol)


@pytest.mark.parametrize("name", list(GRAPHS))
def test_traversals_match(gold, name):
    graph = GRAPHS[name]()
    for ordering in ("dfs", "bfs"):
        ours = [repr(el.id) for el in graph.get_traversal_iterator(ordering=ordering)]
        assert ours == [str(x) for x in gold[f"{name}/traversal_{ordering}"]]
    assert [repr(el.id) for el in graph.get_traversal_iterator()] == [str(x) for x in gold[f"{name}/traversal_bfs"]]


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("ordering", ["dfs", "bfs"])
@pytest.mark.parametrize("sync", [False, True])
def test_bp_sweeps_match(gold, name, ordering, sync):
    graph = GRAPHS[name]()
    tensors = keyed(graph, unpack(gold, f"{name}/tensors"))
    m = keyed(graph, unpack(gold, f"{name}/messages"))
    bp = OM.get_belief_propagation_map(list(graph.get_traversal_iterator(ordering=ordering)), sync)
    for _ in range(2):
        m = bp(tensors, m)
    close_dicts(m, unpack(gold, f"{name}/bp2_{ordering}_{'sync' if sync else 'async'}"), 1e-12)


@pytest.mark.parametrize("name", list(GRAPHS))
def test_gauges_distances_and_densities_match(gold, name):
    graph = GRAPHS[name]()
    trav = list(graph.get_traversal_iterator())
    tensors = keyed(graph, unpack(gold, f"{name}/tensors"))
    m0 = keyed(graph, unpack(gold, f"{name}/messages"))
    bp = OM.get_belief_propagation_map(trav)
    m = m0
    for _ in range(30):
        m = bp(tensors, m)
    close_dicts(m, unpack(gold, f"{name}/messages_30"), 1e-10)
    m30 = keyed(graph, unpack(gold, f"{name}/messages_30"))
    close(OM.messages_frob_distance(m30, bp(tensors, m30)), gold[f"{name}/frob_30_31"], 1e-10)
    g_t, lam = OM.get_vidal_gauge_fixing_map(trav, 1e-10)(tensors, m30)
    close_dicts(g_t, unpack(gold, f"{name}/vidal_tensors"), 1e-10)
    close_dicts(lam, {k: v.real for k, v in unpack(gold, f"{name}/vidal_lambdas").items()}, 1e-10)
    gv_t = keyed(graph, unpack(gold, f"{name}/vidal_tensors"))
    gv_l = keyed(graph, unpack(gold, f"{name}/vidal_lambdas"), real=True)
    close(OM.get_vidal_gauge_distance_map(trav, 1e-10)(gv_t, gv_l), gold[f"{name}/vidal_distance"], 1e-10)
    close_dicts(OM.get_symmetric_gauge_fixing_map(trav, 1e-10)(gv_t, gv_l),
                unpack(gold, f"{name}/symmetric_tensors"), 1e-12)
    close_dicts(OM.lambdas2messages(gv_l), unpack(gold, f"{name}/lambda_messages"), 1e-12)
    rho = {el.id: OM.get_one_side_density_matrix(el, tensors, m30) for el in trav if isinstance(el, Node)}
    close_dicts(rho, unpack(gold, f"{name}/density"), 1e-12)


def test_graph_gate_methods_match(gold):
    """TensorGraph.apply1 / apply2_to_vidal_canonical (rank cap, accuracy
    cap, none) / truncate / apply2 from the 2x3x2 lattice's Vidal form, as
    the reference ran them: tensors, lambdas, truncation errors, entropies
    and the bond dimensions the methods leave on the graph."""
    from dequantizer_b200.graph import Edge

    graph = GRAPHS["lat232"]()
    edges = [el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, Edge)]
    tensors = keyed(graph, unpack(gold, "lat232/vidal_tensors"))
    lambdas = keyed(graph, unpack(gold, "lat232/vidal_lambdas"), real=True)
    rx = np.array([[np.cos(0.3), -1j * np.sin(0.3)], [-1j * np.sin(0.3), np.cos(0.3)]])
    cnot = np.eye(4, dtype=complex)[[0, 1, 3, 2]].reshape(2, 2, 2, 2)
    zz = np.diag(np.exp(1j * np.array([0.3, -0.3, -0.3, 0.3]))).reshape(2, 2, 2, 2)
    rnd = gold["ops/gate_rnd"]
    first = next(el for el in graph.get_traversal_iterator(ordering="dfs") if isinstance(el, Node))
    tensors = OM.apply1(graph, first.id, tensors, rx)
    close_dicts(tensors, unpack(gold, "lat232/ops/after_apply1"), 1e-12)
    steps = [(cnot, edges[0], None, 3), (rnd, edges[1], 1e-3, None), (zz, edges[2], None, None)]
    for i, (gate, edge, acc, rank) in enumerate(steps):
        a, b = edge.id
        tensors, lambdas, err, ent = OM.apply2_to_vidal_canonical(graph, a, b, tensors, lambdas, gate, 1e-10, acc,
                                                                  rank)
        close_dicts(tensors, unpack(gold, f"lat232/ops/step{i}_tensors"), 1e-10)
        close_dicts(lambdas, {k: v.real for k, v in unpack(gold, f"lat232/ops/step{i}_lambdas").items()}, 1e-10)
        close(err, gold[f"ops/step{i}_err"], 1e-8)
        close(ent, gold[f"ops/step{i}_entropy"], 1e-10)
        assert [e.dimension for e in edges] == list(gold[f"ops/step{i}_edge_dims"])
    tensors, lambdas = OM.truncate(graph, tensors, lambdas, 1e-2)
    close_dicts(tensors, unpack(gold, "lat232/ops/truncated_tensors"), 1e-10)
    close_dicts(lambdas, {k: v.real for k, v in unpack(gold, "lat232/ops/truncated_lambdas").items()}, 1e-10)
    assert [e.dimension for e in edges] == list(gold["ops/truncated_edge_dims"])
    a, b = edges[3].id
    tensors = OM.apply2(graph, a, b, tensors, rnd, 1e-10)
    close_dicts(tensors, unpack(gold, "lat232/ops/apply2_tensors"), 1e-10)
    assert [e.dimension for e in edges] == list(gold["ops/apply2_edge_dims"])


def test_emulator_matches(gold):
    """The oracle's BPQuantumEmulator against the reference's on the infinite
    heavy-hex cell (key 42, bond <= 4, regauge per layer, three kicked-Ising
    layers; the reference's initial messages drawn as the oracle draws them):
    every qubit's density matrix after each layer and after two measurements,
    the outcomes, truncation errors, entropies and Vidal distances."""
    from dequantizer_b200.graph import Edge
    from oracle.emulator import BPQuantumEmulator as OracleEmulator

    lat = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    trav = list(lat.get_traversal_iterator())
    em = OracleEmulator(lat, 42, 4, lat.edges_number, 1e-7, 100)
    rzz = np.diag(np.exp(np.array([1j, -1j, -1j, 1j]) * np.pi / 4)).reshape(2, 2, 2, 2)
    rx = np.array([[np.cos(0.4), -1j * np.sin(0.4)], [-1j * np.sin(0.4), np.cos(0.4)]])
    nodes = [el.id for el in trav if isinstance(el, Node)]
    assert [repr(n) for n in nodes] == [str(x) for x in gold["emu/nodes"]]
    for layer in range(3):
        for n in nodes:
            em.apply_q1(rx, n)
        for el in trav:
            if isinstance(el, Edge):
                em.apply_q2(rzz, *el.id)
        close(np.stack([em.dens_q1(n) for n in nodes]), gold[f"emu/rho_{layer}"], 1e-10)
    # the reference draws each sample from its key stream, then re-canonicalises
    # with the next seed; the oracle takes the sample as an argument, so the
    # sample's seed is drawn from its generator first to keep both in step
    outcomes = []
    for i in gold["emu/measured"]:
        sample = np.random.default_rng(int(em._rng.integers(0, 2**31 - 1))).uniform(size=(1,))[0]
        outcomes.append(em.measure(nodes[int(i)], sample))
    assert outcomes == list(gold["emu/outcomes"])
    close(np.stack([em.dens_q1(n) for n in nodes]), gold["emu/rho_after_measure"], 1e-10)
    assert len(em.truncation_errors) == len(gold["emu/truncation_errors"])
    assert np.abs(np.array(em.truncation_errors) - gold["emu/truncation_errors"]).max() < 1e-10
    assert np.abs(np.array(em.entropies) - gold["emu/entropies"]).max() < 1e-10
    assert np.abs(np.array(em.after_regauging_vidal_distances) - gold["emu/after_regauging"]).max() < 1e-10
    assert np.abs(np.array(em.truncated_affected_vidal_distances) - gold["emu/truncated_affected"]).max() < 1e-10


def test_annealer_matches(gold):
    """The reference's run_quantum_annealer (first-order steps, get_scheduler)
    against the same loop built from this package's graph, gate and schedule
    functions (workloads.tensor_graph_of, q1_gate, q2_gate, scheduler,
    HADAMARD) on the oracle emulator: the density matrices after every step,
    truncation errors, entropies and Vidal distances after regauging. This
    pins the annealing gate forms and sign conventions."""
    from dequantizer_b200 import workloads as W
    from oracle.emulator import BPQuantumEmulator as OracleEmulator

    energy = W.EnergyFunction(gold["anneal/amps"], gold["anneal/pairs"], gold["anneal/fields"])
    g = W.tensor_graph_of(energy)
    em = OracleEmulator(g, 7, 4, len(energy.coupled_spin_pairs), 1e-7, 100)
    n = g.nodes_number
    deg = {nid: g.get_node(nid).degree for nid in g.nodes}
    for nid in range(n):
        em.apply_q1(W.HADAMARD, nid)
    for step, (mix, coup) in enumerate(W.scheduler(0.2, lambda t: 1 - t, 6)):
        for (a, b), J in zip(energy.coupled_spin_pairs, energy.coupling_amplitudes):
            a, b = int(a), int(b)
            em.apply_q2(W.q2_gate(J, energy.fields[a] / deg[a], energy.fields[b] / deg[b], coup), a, b)
        for nid in range(n):
            em.apply_q1(W.q1_gate(mix), nid)
        close(np.stack([em.dens_q1(i) for i in range(n)]), gold["anneal/rho_history"][step], 1e-10)
    close(np.stack([em.dens_q1(i) for i in range(n)]), gold["anneal/rho"], 1e-10)
    assert np.abs(np.array(em.truncation_errors) - gold["anneal/truncation_errors"]).max() < 1e-10
    assert np.abs(np.array(em.entropies) - gold["anneal/entropies"]).max() < 1e-10
    ref_vd = gold["anneal/after_regauging"]
    assert len(em.after_regauging_vidal_distances) == len(ref_vd)
    assert np.abs(np.array(em.after_regauging_vidal_distances) - ref_vd).max() < 1e-10


def test_exact_emulator_matches(gold):
    """The oracle's dense-state ExactQuantumEmulator against the reference's on
    a 2x3 lattice: a product state, two layers of random one- and two-qubit
    unitaries (densities after each), then two measurements. The reference's
    samples come from its key 5 (two draws per measurement, the second kept
    only to stay in step with the BP emulator); they are recomputed here from
    the same seeded stream."""
    from dequantizer_b200.graph import Edge
    from oracle.emulator import ExactQuantumEmulator

    lat = G.get_nd_lattice([2, 3], 2, 2, True)
    trav = list(lat.get_traversal_iterator())
    nodes = [el.id for el in trav if isinstance(el, Node)]
    edges = [el.id for el in trav if isinstance(el, Edge)]
    assert [repr(n) for n in nodes] == [str(x) for x in gold["exact/nodes"]]
    em = ExactQuantumEmulator(lat)
    em.set_to_product_state({n: int(b) for n, b in zip(nodes, gold["exact/bits"])})
    for layer in range(2):
        for n, g in zip(nodes, gold[f"exact/g1_{layer}"]):
            em.apply_q1(g, n)
        for e, g in zip(edges, gold[f"exact/g2_{layer}"]):
            em.apply_q2(g, e[0], e[1])
        close(np.stack([em.dens_q1(n) for n in nodes]), gold[f"exact/rho_{layer}"], 1e-12)
    stream = np.random.default_rng(5)
    outcomes = []
    for i in gold["exact/measured"]:
        sample = np.random.default_rng(int(stream.integers(0, 2**31 - 1))).uniform(size=(1,))[0]
        stream.integers(0, 2**31 - 1)
        outcomes.append(em.measure(nodes[int(i)], sample))
    assert outcomes == list(gold["exact/outcomes"])
    close(np.stack([em.dens_q1(n) for n in nodes]), gold["exact/rho_after"], 1e-12)
