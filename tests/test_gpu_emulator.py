"""GPU BPQuantumEmulator and BPEngine.

* The reference's emulator test (quantum_emulator/test_bp_quantum_emulator.py:21-108)
  on the GPU emulator, against the dense exact emulator: rho within the
  reference's tolerances (3e-3 heavy cube, 1e-4 heavy hex / tree), identical
  measurement outcomes for shared uniform samples.
* The GPU emulator against the FP64 oracle emulator fed the same seeds:
  same BP schedule (asynchronous DFS) and same random messages, so the
  density matrices agree to 1e-9 and the truncation errors / entropies to 1e-9.
* BPEngine sweeps (sync, async, flooding) against the oracle.
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import BPQuantumEmulator
from dequantizer_b200 import graph as G
from dequantizer_b200.engine import BPEngine
from dequantizer_b200.graph import MessageID, Node
from oracle import maps as OM
from oracle import tensor_ops as OT
from oracle.emulator import BPQuantumEmulator as OracleEmulator
from oracle.emulator import ExactQuantumEmulator
from tests.helpers import heavy_cube, random_ising_q2_gate, random_q1_gate, random_tensors, rel_err, small_heavy_hex, to_np

pytestmark = pytest.mark.gpu


def _run(graph_factory, layers, accuracy, seed=42, compare_oracle=True):
    rng = np.random.default_rng(seed)
    g_gpu, g_exact, g_orc = graph_factory(), graph_factory(), graph_factory()
    trav = list(g_gpu.get_traversal_iterator())
    exact = ExactQuantumEmulator(g_exact)
    gpu = BPQuantumEmulator(g_gpu, seed, 1024, g_gpu.edges_number, belief_propagation_accuracy=1e-6)
    orc = OracleEmulator(g_orc, seed, 1024, g_orc.edges_number, belief_propagation_accuracy=1e-6) if compare_oracle else None
    nodes = [el for el in trav if isinstance(el, Node)]
    state = {n.id: int(rng.integers(0, 2)) for n in nodes}
    exact.set_to_product_state(state)
    gpu.set_to_product_state(state)
    if orc:
        orc.set_to_product_state(state)
    for nid, s in state.items():
        correct = np.zeros((2, 2))
        correct[s, s] = 1.0
        assert np.isclose(to_np(gpu.dens_q1(nid)), correct, atol=1e-8).all()
        u = float(rng.uniform())
        assert gpu.measure(nid, u) == s
        if orc:
            assert orc.measure(nid, u) == s
    for _ in range(layers):
        for el in trav:
            if isinstance(el, Node):
                g = random_q1_gate(rng)
                for em in (exact, gpu, orc):
                    if em is not None:
                        em.apply_q1(g, el.id)
            else:
                g = random_ising_q2_gate(rng)
                for em in (exact, gpu, orc):
                    if em is not None:
                        em.apply_q2(g, *el.id)
    for el in nodes:
        rho_g = to_np(gpu.dens_q1(el.id))
        assert np.linalg.norm(exact.dens_q1(el.id) - rho_g) < accuracy
        if orc:
            assert np.abs(orc.dens_q1(el.id) - rho_g).max() < 1e-9
    if orc:
        te_g = np.array([float(x) for x in gpu.truncation_errors])
        en_g = np.array([float(x) for x in gpu.entropies])
        assert len(te_g) == len(orc.truncation_errors)
        assert np.abs(te_g - np.array(orc.truncation_errors)).max() < 1e-9
        assert np.abs(en_g - np.array(orc.entropies)).max() < 1e-9
        assert gpu.bp_iterations == orc.bp_iterations
    for el in nodes:
        u = float(rng.uniform())
        assert exact.measure(el.id, u) == gpu.measure(el.id, u)


def test_gpu_emulator_heavy_cube():
    _run(heavy_cube, 2, 3e-3)


def test_gpu_emulator_small_heavy_hex():
    _run(small_heavy_hex, 4, 1e-4)


def test_gpu_emulator_random_tree():
    _run(lambda: G.get_random_tree_tensor_graph(15, 2, 14 * [1], 42), 4, 1e-4)


def test_emulator_regauges_per_reference_rule():
    g = heavy_cube()
    em = BPQuantumEmulator(g, 3, 8, 5, belief_propagation_accuracy=1e-6)
    rng = np.random.default_rng(0)
    edges = list(g.edges)
    for i in range(12):
        em.apply_q2(random_ising_q2_gate(rng), *edges[i])
    # regauge before gates 6 and 11 -> two truncation-affected distances
    assert len(em.truncated_affected_vidal_distances) == 2
    assert len(em.truncation_errors) == 12
    assert all(e.dimension <= 8 for e in g.edges.values())


@pytest.mark.parametrize("chi", [8, 16])
def test_engine_fp32_sweeps_track_fp64(chi):
    """complex64 sweeps (FP32 arithmetic) stay within FP32 rounding of the
    complex128 sweeps from the same start; tolerance 1e-5 relative."""
    g = G.get_random_regular_graph(32, 3, 2, chi, 9)
    tensors = random_tensors(g, 5)
    e64 = BPEngine(g, schedule="sync", precision="fp64")
    e32 = BPEngine(g, schedule="sync", precision="fp32")
    order = [tensors[n.id] / np.linalg.norm(tensors[n.id]) for n in e64.topo.nodes]
    rng = np.random.default_rng(6)
    mats = []
    for h in range(e64.layout.n_halves):
        z = rng.standard_normal((chi, chi, 2))
        a = z[..., 0] + 1j * z[..., 1]
        m = a @ a.conj().T
        mats.append(m / np.trace(m).real)
    for e in (e64, e32):
        e.load_tensors(order)
        e.load_messages(mats)
    for _ in range(5):
        e64.sweep()
        e32.sweep()
    a = e64.n2e
    b = e32.n2e.to(torch.complex128)
    assert float((a - b).abs().max() / a.abs().max()) < 1e-5
    e32.check()


def _bench_like(n, seed, chi=16):
    g = G.get_random_regular_graph(n, 3, 2, chi, seed)
    rng = np.random.default_rng(seed + 100)
    tensors = []
    for _ in range(n):
        z = rng.standard_normal((chi**3 * 2, 2))
        tensors.append((z[:, 0] + 1j * z[:, 1]) / np.sqrt(2 * 2 * chi**3))
    a = rng.standard_normal((chi, chi, 2))
    a = a[..., 0] + 1j * a[..., 1]
    m = a @ a.conj().T
    return g, tensors, m / np.trace(m).real


def test_engine_bf16_sweeps_track_fp64():
    """BF16 tensor-core sweeps from the same start stay within BF16 operand
    rounding (relative 3e-2 per message entry) of the FP64 sweeps."""
    g, tensors, m = _bench_like(48, 3)
    engines = {p: BPEngine(g, schedule="sync", precision=p) for p in ("fp64", "bf16")}
    for e in engines.values():
        e.load_tensors(tensors)
        e.load_messages([m] * e.layout.n_halves)
    for _ in range(4):
        for e in engines.values():
            e.sweep()
    a = engines["fp64"].n2e
    b = engines["bf16"].n2e.to(torch.complex128)
    assert float((a - b).abs().max() / a.abs().max()) < 3e-2
    engines["bf16"].check()


@pytest.mark.parametrize("schedule", ["sync", "async"])
def test_bf16_tcgen05_kernel_matches_mma_sync_kernel(schedule):
    """The tcgen05 node update (mode products in tensor memory) and the
    warp-MMA one round the same intermediates to BF16 and accumulate in FP32:
    after one and after three sweeps from the same start their messages agree
    to 1e-2 of the largest entry (FP32 summation order moves BF16 roundings),
    both stay within 3e-2 of FP64, and no node is skipped."""
    g, tensors, m = _bench_like(40, 11)
    engines = {k: BPEngine(g, schedule=schedule, precision="bf16", bf16_kernel=k) for k in ("tcgen05", "mma_sync")}
    ref = BPEngine(g, schedule=schedule, precision="fp64")
    for e in list(engines.values()) + [ref]:
        e.load_tensors(tensors)
        e.load_messages([m] * e.layout.n_halves)
    assert engines["tcgen05"].kernel == "bp_node_k3_umma"
    for n_sweeps in (1, 2):
        for e in list(engines.values()) + [ref]:
            for _ in range(n_sweeps):
                e.sweep()
        a = engines["tcgen05"].n2e.to(torch.complex128)
        b = engines["mma_sync"].n2e.to(torch.complex128)
        assert bool(torch.isfinite(a).all())
        assert float((a - b).abs().max() / b.abs().max()) < 1e-2
        assert float((a - ref.n2e).abs().max() / ref.n2e.abs().max()) < 3e-2
    for e in engines.values():
        e.check()


def test_engine_bf16_meets_z_bound_at_fixed_point():
    """<Z_i> after BP to the fixed point: BF16 sweeps vs FP64 sweeps,
    |delta <Z_i>| <= 1e-4 (the mixed-precision accuracy bound)."""
    g, tensors, m = _bench_like(96, 5)
    z = {}
    for p in ("fp64", "bf16", "fp32"):
        e = BPEngine(g, schedule="sync", precision=p)
        e.load_tensors(tensors)
        e.load_messages([m] * e.layout.n_halves)
        for _ in range(80):
            e.sweep()
        rho = to_np(e.densities())
        z[p] = (rho[:, 0, 0] - rho[:, 1, 1]).real
    assert np.abs(z["fp32"] - z["fp64"]).max() < 1e-6
    assert np.abs(z["bf16"] - z["fp64"]).max() < 1e-4


@pytest.mark.parametrize("precision,schedule", [("fp64", "async"), ("fp64", "sync"), ("bf16", "sync")])
def test_graphed_sweeps_equal_eager_sweeps(precision, schedule):
    """run_graphed replays captured blocks of sweeps: after the same number
    of sweeps the messages equal the eager engine's bit for bit."""
    g, tensors, m = _bench_like(24, 8)
    engines = [BPEngine(g, schedule=schedule, precision=precision) for _ in range(2)]
    for e in engines:
        e.load_tensors(tensors)
        e.load_messages([m] * e.layout.n_halves)
    n = engines[1].run_graphed(0.0, max_sweeps=2 + 4 * 3, block=4)
    assert n == 14
    for _ in range(n):
        engines[0].sweep()
    assert torch.equal(engines[0].n2e, engines[1].n2e)
    assert torch.equal(engines[0].e2n, engines[1].e2n)


@pytest.mark.parametrize("schedule", ["sync", "async", "flooding"])
def test_engine_sweeps_match_oracle(schedule):
    g = G.get_random_regular_graph(16, 3, 2, 4, 5)
    eng = BPEngine(g, traversal="dfs", schedule=schedule)
    trav = eng.topo.traverser
    tensors = random_tensors(g, 1)
    rng = np.random.default_rng(2)
    L = eng.layout
    eng.load_tensors([tensors[n.id] for n in eng.topo.nodes])
    mats = []
    for h in range(L.n_halves):
        z = rng.standard_normal((4, 4, 2))
        a = z[..., 0] + 1j * z[..., 1]
        mats.append(a @ a.conj().T)
    e2n = []
    for h in range(L.n_halves):
        e2n.append(mats[int(L.half_twin[h])])
    eng.load_messages(mats, e2n)
    # oracle messages dict matching the packed state
    msgs = {}
    for h, (nd, e) in enumerate(eng.topo.half_ids()):
        msgs[MessageID(nd.id, e.id)] = mats[h]
        msgs[MessageID(e.id, nd.id)] = e2n[h]
    if schedule == "flooding":
        # node update reads the far end's previous node->edge message directly
        def ref_sweep(t, m):
            out = {}
            for nd in eng.topo.nodes:
                inc = [m[MessageID(e.neighbors[1].id if e.neighbors[0] is nd else e.neighbors[0].id, e.id)]
                       for e in nd.neighbors]
                new = OT.pass_through_node(t[nd.id], inc)
                for e, x in zip(nd.neighbors, new):
                    out[MessageID(nd.id, e.id)] = x
            for nd in eng.topo.nodes:
                for e in nd.neighbors:
                    u = e.neighbors[1] if e.neighbors[0] is nd else e.neighbors[0]
                    out[MessageID(e.id, nd.id)] = out[MessageID(u.id, e.id)]
            return out
    else:
        ref_sweep = OM.get_belief_propagation_map(trav, schedule == "sync")
    for _ in range(4):
        msgs = ref_sweep(tensors, msgs)
        eng.sweep()
    for h, (nd, e) in enumerate(eng.topo.half_ids()):
        assert rel_err(L.message_view(eng.n2e, h), msgs[MessageID(nd.id, e.id)]) < 1e-11
        assert rel_err(L.message_view(eng.e2n, h), msgs[MessageID(e.id, nd.id)]) < 1e-11
    iters = eng.run(1e-12, max_sweeps=300)
    assert iters < 300
    G_, lam = eng.vidal_gauge()
    vd = float(eng.vidal_distance(G_, lam))
    assert vd < 1e-8
    rho = to_np(eng.densities())
    assert np.allclose(np.trace(rho, axis1=1, axis2=2), 1.0)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "bf16"])
def test_pipelined_host_sweep_equals_plain_sequence(precision):
    """BPEngine.sweep_host (uploads in node ranges overlapped with the
    per-range node updates and downloads) gives the plain load / sweep /
    read-back sequence bit for bit, twice in a row."""
    from dequantizer_b200.engine import BPEngine
    from dequantizer_b200.graph import get_random_regular_graph

    g = get_random_regular_graph(40, 3, 2, 16, 2)
    rng = np.random.default_rng(3)
    engs = [BPEngine(g, schedule="sync", precision=precision) for _ in range(2)]
    L = engs[0].layout
    mdt = torch.complex128 if precision == "fp64" else torch.complex64
    outs = [[], []]
    for step in range(2):
        z = rng.standard_normal((L.tensor_elems, 2)) / 64
        packed = torch.from_numpy(z[:, 0] + 1j * z[:, 1]).to(torch.complex64).pin_memory()
        a = rng.standard_normal((L.msg_elems, 2))
        n2e = torch.from_numpy(a[:, 0] + 1j * a[:, 1]).to(mdt).pin_memory()
        e2n = torch.from_numpy(a[::-1, 1] + 1j * a[::-1, 0]).to(mdt).pin_memory()
        for k, eng in enumerate(engs):
            out = torch.empty_like(n2e).pin_memory()
            if k == 0:
                eng.load_tensors_host(packed)
                eng.load_messages_host(n2e, e2n)
                eng.sweep()
                eng.read_messages_host(out)
            else:
                eng.sweep_host(packed, n2e, e2n, out, chunks=5)
            torch.cuda.synchronize()
            outs[k].append(out.clone())
        assert torch.equal(outs[0][step], outs[1][step])
        assert torch.equal(engs[0].e2n, engs[1].e2n)
    engs[1].check()
