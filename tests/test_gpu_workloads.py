"""The example workloads on the GPU against the same loops run on the oracle.

* 3-D Ising square-root network (examples/3d_ising_canonicalization.py:89-160):
  same Vidal-distance history, iteration count and magnetisation.
* Kicked Ising on the infinite heavy-hex cell (examples/ibm_eagle_processor.py:56-145).
* Quantum annealing, first- and second-order Trotter steps
  (examples/quantum_annealing/quantum_annealing/src/quantum_annealer.py:90-152).
Tolerances: 1e-9 on magnetisations / <Z> / density matrices (FP64 on both
sides, the same BP schedule and the same seeded messages).
"""

import numpy as np
import pytest
import torch

from dequantizer_b200 import workloads as W
from dequantizer_b200 import graph as G
from dequantizer_b200 import maps as M
from dequantizer_b200.graph import Edge, Node
from dequantizer_b200.initializers import get_message_random_nonnegative_initializer, get_potts_initializer
from oracle import maps as OM
from oracle.emulator import BPQuantumEmulator as OracleEmulator

pytestmark = pytest.mark.gpu


def oracle_ising(sizes, betas, coupling, field, accuracy, key=42):
    lat = G.get_nd_lattice(list(sizes), 2, 2, True)
    trav = list(lat.get_traversal_iterator(ordering="dfs"))
    bp = OM.get_belief_propagation_map(trav)
    vg = OM.get_vidal_gauge_fixing_map(trav, accuracy)
    vd = OM.get_vidal_gauge_distance_map(trav, accuracy)
    spins = np.array([1.0, -1.0])
    out = []
    for beta in betas:
        init = get_potts_initializer(np.exp(-coupling * beta * np.tensordot(spins, spins, axes=0)),
                                     np.exp(-field * beta * spins))
        tensors = OM.init_tensors(lat, init)
        msgs = lat.init_messages(get_message_random_nonnegative_initializer(key))
        hist, d = [], np.finfo(np.float64).max
        while d > accuracy:
            msgs = bp(tensors, msgs)
            t, l = vg(tensors, msgs)
            d = vd(t, l)
            hist.append(d)
        mag = np.mean([2 * OM.get_one_side_density_matrix(el, tensors, msgs)[0, 0].real - 1
                       for el in trav if isinstance(el, Node)])
        out.append((hist, mag))
    return out


@pytest.mark.parametrize("field", [0.5, 0.0])
def test_ising_sqrt_partition_matches_oracle(field):
    betas = [0.1, 0.4]
    res = W.ising_sqrt_partition([3, 3, 3], betas, coupling=-1.0, field_strength=field, accuracy=1e-9)
    ref = oracle_ising([3, 3, 3], betas, -1.0, field, 1e-9)
    for i, (hist, mag) in enumerate(ref):
        assert res.number_of_iterations[i] == len(hist)
        assert np.abs(res.vidal_dist_per_iter[i] - np.array(hist)).max() < 1e-9
        assert abs(res.average_magnetization[i] - mag) < 1e-9


@pytest.mark.parametrize("sync", [False, True])
def test_graphed_canonicalisation_equals_eager(sync):
    """BPEngine.canonicalise with graph replays (one graph per buffer
    assignment) gives the eager loop's distances, lambdas, final messages and
    densities bit for bit, at two stopping tolerances (different replay counts)."""
    from dequantizer_b200.engine import BPEngine

    lat = G.get_nd_lattice([4, 4, 3], 2, 2, True)
    spins = np.array([1.0, -1.0])
    init = get_potts_initializer(np.exp(0.3 * np.tensordot(spins, spins, axes=0)), np.exp(-0.15 * spins))
    runs = {}
    for graphed in (False, True):
        for tol in (1e-10, 3e-11):  # two stopping points, so the replay counts differ
            eng = BPEngine(lat, traversal="dfs", schedule="sync" if sync else "async")
            eng.load_tensors([init(n) for n in eng.topo.nodes])
            mi = get_message_random_nonnegative_initializer(42)
            eng.load_messages([mi((nd, e)) for nd, e in eng.topo.half_ids()],
                              [mi((e, nd)) for nd, e in eng.topo.half_ids()])
            hist, Gm, lam = eng.canonicalise(tol, 500, graphed=graphed)
            runs[(graphed, tol)] = (hist, lam.clone(), eng.n2e.clone(), eng.densities().clone())
    for tol in (1e-10, 3e-11):
        a, b = runs[(False, tol)], runs[(True, tol)]
        assert len(a[0]) > 3 and a[0] == b[0]
        for x, y in zip(a[1:], b[1:]):
            assert torch.equal(x, y)
    # the same engine on reloaded inputs replays its cached graphs from the first iteration
    eng = BPEngine(lat, traversal="dfs", schedule="sync" if sync else "async")
    for rep in range(2):
        eng.load_tensors([init(n) for n in eng.topo.nodes])
        mi = get_message_random_nonnegative_initializer(42)
        eng.load_messages([mi((nd, e)) for nd, e in eng.topo.half_ids()],
                          [mi((e, nd)) for nd, e in eng.topo.half_ids()])
        hist, Gm, lam = eng.canonicalise(1e-10, 500, graphed=True)
        assert hist == runs[(False, 1e-10)][0]
        assert torch.equal(lam, runs[(False, 1e-10)][1])
        assert torch.equal(eng.densities(), runs[(False, 1e-10)][3])


def test_kicked_ising_infinite_cell_matches_oracle():
    z_gpu, _ = W.run_eagle_simulation(max_chi=8, layers_per_regauging=1, trotter_steps=3, accuracy=1e-7,
                                      theta=0.8, is_infinite=True, max_belief_propagation_iterations=100)
    lat = G.get_heavy_hex_ibm_eagle_lattice_infinite()
    trav = list(lat.get_traversal_iterator())
    em = OracleEmulator(lat, 42, 8, lat.edges_number, 1e-7, 100)
    rzz, rx = W.kicked_ising_gates(0.8)
    z_ref = [float((em.dens_q1(2)[0, 0] - em.dens_q1(2)[1, 1]).real)]
    for _ in range(3):
        for nid in range(lat.nodes_number):
            em.apply_q1(rx, nid)
        for el in trav:
            if isinstance(el, Edge):
                em.apply_q2(rzz, *el.id)
        rho = em.dens_q1(2)
        z_ref.append(float((rho[0, 0] - rho[1, 1]).real))
    assert np.abs(np.array(z_gpu) - np.array(z_ref)).max() < 1e-9


@pytest.mark.parametrize("second_order", [False, True])
def test_annealing_matches_oracle(second_order):
    energy = W.random_regular_energy(10, 3, seed=4, field_std=0.5)
    steps = list(W.scheduler(0.2, lambda t: 1 - t, 6))
    res = W.run_quantum_annealer(energy, steps, key=7, max_chi=4, gates_number_per_regauging=energy.edges_number,
                                 accuracy=1e-7, max_belief_propagation_iterations=100,
                                 second_order=second_order)
    g = W.tensor_graph_of(energy)
    em = OracleEmulator(g, 7, 4, energy.edges_number, 1e-7, 100)
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
    rho_ref = np.stack([em.dens_q1(i) for i in range(n)])
    assert np.abs(res.density_matrices - rho_ref).max() < 1e-9
    assert np.abs(res.truncation_errors - np.array(em.truncation_errors)).max() < 1e-9
    assert np.abs(res.entropies - np.array(em.entropies)).max() < 1e-9
    assert np.abs(res.vidal_distances_after_regauging - np.array(em.after_regauging_vidal_distances)).max() < 1e-9
    spins = 2 * (res.density_matrices[:, 0, 0].real > 0.5) - 1
    assert np.isfinite(W.eval_energy(energy, spins))


def test_batched_annealer_equals_independent_runs():
    """Instances advanced together (one launch per operation over all of
    them) give the same density matrices and truncation errors as separate
    runs of the emulator loop (synchronous BP schedule on both sides)."""
    from dequantizer_b200.annealing import BatchedAnnealer

    energies = [W.random_regular_energy(n, 3, seed=10 + n, field_std=0.5) for n in (8, 10, 12)]
    steps = list(W.scheduler(0.2, lambda t: 1 - t, 5))
    ba = BatchedAnnealer(energies, max_chi=4, accuracy=1e-8, max_belief_propagation_iterations=100)
    rho_b = ba.run(steps)
    errs_b = ba.truncation_errors()
    for k, en in enumerate(energies):
        res = W.run_quantum_annealer(en, steps, key=1, max_chi=4, gates_number_per_regauging=en.edges_number,
                                     accuracy=1e-8, max_belief_propagation_iterations=100,
                                     synchronous_update=True)
        assert np.abs(rho_b[k] - res.density_matrices).max() < 1e-9
        assert np.abs(errs_b[k] - res.truncation_errors).max() < 1e-9


def test_batched_measurement_sampling_equals_independent_runs():
    """Measuring every qubit after annealing (quantum_annealer.py:137-141):
    the batched annealer, all instances per round, gives the same outcomes as
    the emulator loop of each instance fed the same uniform draws."""
    from dequantizer_b200.annealing import BatchedAnnealer

    energies = [W.random_regular_energy(n, 3, seed=30 + n, field_std=0.5) for n in (8, 10)]
    steps = list(W.scheduler(0.2, lambda t: 1 - t, 4))
    U = np.random.default_rng(5).uniform(size=(2, 10))
    ba = BatchedAnnealer(energies, max_chi=4, accuracy=1e-10, max_belief_propagation_iterations=200)
    ba.run(steps)
    spin_configs = ba.sample_measurements(samples=U)
    for k, en in enumerate(energies):
        res = W.run_quantum_annealer(en, steps, key=1, max_chi=4, gates_number_per_regauging=en.edges_number,
                                     accuracy=1e-10, max_belief_propagation_iterations=200,
                                     synchronous_update=True, sample_measurements=True, samples=U[k])
        assert np.array_equal(spin_configs[k], res.configuration)
        assert set(np.unique(spin_configs[k])) <= {-1, 1}


def test_mixed_precision_batched_annealer_tracks_fp64():
    """BatchedAnnealer(precision="mixed"): once every bond has dimension 16,
    each regauge starts with BF16 tensor-core sweeps, then FP32 sweeps, and
    hands over to the FP64 loop of the reference; the densities stay within
    1e-4 of the FP64 annealer's (the FP64 loop finishes every regauge to the
    same accuracy)."""
    from dequantizer_b200.annealing import BatchedAnnealer

    energies = [W.random_regular_energy(n, 3, seed=60 + n, field_std=0.5) for n in (16, 20, 24)]
    steps = list(W.scheduler(0.5, lambda t: 1 - t, 10))
    runs = {}
    for prec in ("fp64", "mixed"):
        ba = BatchedAnnealer(energies, max_chi=16, accuracy=1e-7, max_belief_propagation_iterations=200,
                             precision=prec)
        runs[prec] = (ba.run(steps, second_order=True), ba)
    mixed = runs["mixed"][1]
    assert mixed.layout.uniform_k3_chi() == 16
    assert sum(sum(s) for s in mixed.bf16_sweeps) > 0, "no regauge took the BF16 path"
    assert sum(sum(s) for s in mixed.fp32_sweeps) > 0, "no regauge took the FP32 stage"
    for k in range(len(energies)):
        assert np.abs(runs["mixed"][0][k] - runs["fp64"][0][k]).max() < 1e-4
    assert int(M.error_flag(torch.device("cuda", 0)).item()) == 0
