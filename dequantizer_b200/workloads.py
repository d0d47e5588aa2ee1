"""Drivers of the reference's example workloads on the GPU path.

* ``ising_sqrt_partition``  -- examples/3d_ising_canonicalization.py:89-160:
  square-root Ising partition-function network on an N-d lattice, BP + Vidal
  gauge + Vidal distance per iteration until the distance reaches the
  accuracy, then the average magnetisation from the one-site density
  matrices (2 rho_00 - 1).
* ``run_eagle_simulation``  -- examples/ibm_eagle_processor.py:56-145:
  kicked Ising (RX(theta) on every qubit, RZZ(-pi/2) on every edge) with the
  BP emulator; returns <Z> of a target qubit per layer, or of all qubits.
* ``run_quantum_annealer``  -- examples/quantum_annealing/quantum_annealing/src/
  quantum_annealer.py:90-152 with ``scheduler`` (scheduler.py:7-14) and the
  gate builders (:44-84); ``second_order=True`` applies a Strang step
  (half mixing, full coupling, half mixing) instead of the reference's
  first-order step.
"""

from dataclasses import dataclass, field
from typing import Callable, Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .emulator import BPQuantumEmulator
from .engine import BPEngine
from .graph import Edge, Node, TensorGraph, get_heavy_hex_ibm_eagle_lattice, get_heavy_hex_ibm_eagle_lattice_infinite
from .graph import get_nd_lattice, greedy_edge_coloring
from .initializers import get_message_random_nonnegative_initializer, get_potts_initializer

HADAMARD = np.sqrt(0.5) * np.array([[1, 1], [1, -1]], dtype=np.complex128)


# ------------------------------------------------ 3-D Ising square-root network
@dataclass
class CanonicalizationResult:
    vidal_dist_per_iter: List[np.ndarray] = field(default_factory=list)
    number_of_iterations: List[int] = field(default_factory=list)
    average_magnetization: List[float] = field(default_factory=list)
    lambdas: List[torch.Tensor] = field(default_factory=list)


def ising_sqrt_partition(
    lattice_sizes: Sequence[int],
    betas: Iterable[float],
    coupling: float,
    field_strength: float,
    accuracy: float,
    open_boundary: bool = True,
    synchronous_update: bool = False,
    key: int = 42,
    traversal_type: str = "dfs",
    max_iterations: int = 500,
    graphed: bool = False,
) -> CanonicalizationResult:
    """BP + Vidal gauge on the square-root Ising network for each beta
    (bond dimension 2, physical dimension 2, FP64). ``graphed`` replays each
    iteration (sweep, gauge, distance) as a CUDA graph (BPEngine.canonicalise);
    the results are the eager loop's. It is off by default: on the 6x6x6
    lattice an iteration is a chain of ~200 dependent level launches whose
    device-side latency a graph does not remove, and capturing costs more than
    replay saves over one scan."""
    lattice = get_nd_lattice(list(lattice_sizes), 2, 2, open_boundary)
    eng = BPEngine(lattice, traversal=traversal_type, schedule="sync" if synchronous_update else "async")
    L = eng.layout
    res = CanonicalizationResult()
    spins = np.array([1.0, -1.0])
    for beta in betas:
        two = np.exp(-coupling * beta * np.tensordot(spins, spins, axes=0))
        one = np.exp(-field_strength * beta * spins)
        init = get_potts_initializer(two, one)
        eng.load_tensors([init(n) for n in eng.topo.nodes])
        msg_init = get_message_random_nonnegative_initializer(key)
        n2e = [msg_init((nd, e)) for nd, e in eng.topo.half_ids()]
        e2n = [msg_init((e, nd)) for nd, e in eng.topo.half_ids()]
        eng.load_messages(n2e, e2n)
        hist, G, lam = eng.canonicalise(accuracy, max_iterations, graphed=graphed)
        rho = eng.densities()
        mag = float((2 * rho[:, 0, 0].real - 1).mean())
        res.vidal_dist_per_iter.append(np.array(hist))
        res.number_of_iterations.append(len(hist))
        res.average_magnetization.append(mag)
        res.lambdas.append(lam)
    return res


# ---------------------------------------------- kicked Ising, heavy-hex lattice
def kicked_ising_gates(theta: float):
    """RZZ(-pi/2) and RX(theta) (ibm_eagle_processor.py:97-118)."""
    rzz = np.diag(np.exp(np.array([1j, -1j, -1j, 1j]) * np.pi / 4)).reshape((2, 2, 2, 2))
    rx = np.array([[np.cos(theta / 2), -1j * np.sin(theta / 2)], [-1j * np.sin(theta / 2), np.cos(theta / 2)]],
                  dtype=np.complex128)
    return rzz, rx


def run_eagle_simulation(
    max_chi: int,
    layers_per_regauging: int,
    trotter_steps: int,
    accuracy: float,
    theta: float,
    is_infinite: bool = True,
    synchronous_update: bool = False,
    max_belief_propagation_iterations: Optional[int] = None,
    key: int = 42,
    traversal_type: str = "dfs",
    colour_classes: bool = False,
    all_qubits: bool = False,
    on_step: Optional[Callable[[int], None]] = None,
):
    """Kicked-Ising dynamics; returns the target qubit's <Z> per layer (layer 0
    first), or every qubit's <Z> per layer when ``all_qubits``. With
    ``colour_classes`` the RZZ gates are applied class by class of a proper
    edge colouring with a regauge after each class. ``on_step(t)`` is called
    before Trotter step t and with t = trotter_steps after the last one."""
    lattice = get_heavy_hex_ibm_eagle_lattice_infinite() if is_infinite else get_heavy_hex_ibm_eagle_lattice()
    traverser = list(lattice.get_traversal_iterator())
    target = 2 if is_infinite else 62
    classes = greedy_edge_coloring(lattice) if colour_classes else None
    per_regauging = (max(len(c) for c in classes) if classes else lattice.edges_number * layers_per_regauging)
    em = BPQuantumEmulator(lattice, key, max_chi, per_regauging, accuracy, max_belief_propagation_iterations,
                           synchronous_update, traversal_type)
    rzz, rx = kicked_ising_gates(theta)

    def readout():
        if all_qubits:
            rho = em.all_densities()
            return (rho[:, 0, 0] - rho[:, 1, 1]).real.cpu().numpy()
        rho = em.dens_q1(target)
        return float((rho[0, 0] - rho[1, 1]).real)

    out = [readout()]
    for t in range(trotter_steps):
        if on_step is not None:
            on_step(t)
        for node_id in range(lattice.nodes_number):
            em.apply_q1(rx, node_id)
        if classes:
            for cls in classes:
                for eid in cls:
                    em.apply_q2(rzz, eid[0], eid[1])
                em._vidal_regauging()
                em._passed = 0
        else:
            for el in traverser:
                if isinstance(el, Edge):
                    em.apply_q2(rzz, el.id[0], el.id[1])
        out.append(readout())
    if on_step is not None:
        on_step(trotter_steps)
    return out, em


# ----------------------------------------------------------- quantum annealing
@dataclass
class EnergyFunction:
    """J_ij on coupled pairs and fields h_i (energy_function.py)."""

    coupling_amplitudes: np.ndarray
    coupled_spin_pairs: np.ndarray
    fields: np.ndarray

    @property
    def edges_number(self) -> int:
        return int(self.coupled_spin_pairs.shape[0])


def random_regular_energy(nodes_number: int, degree: int, seed: int, field_std: float = 0.0,
                          pm_one: bool = True) -> EnergyFunction:
    """Random regular instance: pairing-model graph, J = +-1 uniform (or
    normal), h normal * field_std."""
    from .graph import random_regular_pairs

    rng = np.random.default_rng(seed)
    pairs = np.array(random_regular_pairs(nodes_number, degree, seed), dtype=np.int64)
    if pm_one:
        J = rng.choice(np.array([-1.0, 1.0]), size=len(pairs))
    else:
        J = rng.standard_normal(len(pairs))
    h = rng.standard_normal(nodes_number) * field_std
    return EnergyFunction(J, pairs, h)


def scheduler(total_time_step_size: float, schedule, steps_number: int):
    """scheduler.py:7-14: yields (mixing_time, coupling_time)."""
    for i in range(steps_number):
        f = schedule(i / (steps_number - 1))
        yield total_time_step_size * f, total_time_step_size * (1 - f)


def q2_gate(J: float, h1_over_deg: float, h2_over_deg: float, tau: float) -> np.ndarray:
    """exp(-i tau (J ZZ + h1/deg1 Z1 + h2/deg2 Z2)), diagonal (quantum_annealer.py:59-68)."""
    ham = (J * np.array([1, -1, -1, 1], dtype=np.complex128)
           + h1_over_deg * np.array([1, 1, -1, -1], dtype=np.complex128)
           + h2_over_deg * np.array([1, -1, 1, -1], dtype=np.complex128))
    return np.diag(np.exp(-1j * tau * ham)).reshape((2, 2, 2, 2))


def q1_gate(tau: float) -> np.ndarray:
    """exp(-i tau X) (quantum_annealer.py:72-84)."""
    return np.array([[np.cos(tau), -1j * np.sin(tau)], [-1j * np.sin(tau), np.cos(tau)]], dtype=np.complex128)


@dataclass
class QuantumAnnealingResults:
    density_matrices: np.ndarray
    vidal_distances_after_regauging: np.ndarray
    truncation_affected_vidal_distances: np.ndarray
    truncation_errors: np.ndarray
    entropies: np.ndarray
    configuration: Optional[np.ndarray] = None


def tensor_graph_of(energy: EnergyFunction) -> TensorGraph:
    """quantum_annealer.py:34-41."""
    g = TensorGraph()
    for i in range(energy.fields.shape[0]):
        g.add_node(2, i)
    for a, b in energy.coupled_spin_pairs:
        g.add_edge((int(a), int(b)), 1)
    return g


def run_quantum_annealer(
    energy: EnergyFunction,
    schedule_iter: Iterable[Tuple[float, float]],
    key: int,
    max_chi: int,
    gates_number_per_regauging: int,
    accuracy: float,
    max_belief_propagation_iterations: Optional[int],
    synchronous_update: bool = False,
    traversal_type: str = "dfs",
    second_order: bool = False,
    sample_measurements: bool = False,
    samples: Optional[Sequence[float]] = None,
) -> QuantumAnnealingResults:
    """Annealing on the BP emulator (quantum_annealer.py:90-152). With
    ``sample_measurements`` every qubit is then measured in node order
    (quantum_annealer.py:137-141) and ``configuration`` = 1 - 2 * outcomes;
    ``samples`` (one uniform draw per qubit) replaces the emulator's own draws."""
    g = tensor_graph_of(energy)
    em = BPQuantumEmulator(g, key, max_chi, gates_number_per_regauging, accuracy,
                           max_belief_propagation_iterations, synchronous_update, traversal_type)
    n = g.nodes_number
    deg = {nid: g.get_node(nid).degree for nid in g.nodes}
    for nid in range(n):
        em.apply_q1(HADAMARD, nid)
    for mixing_time, coupling_time in schedule_iter:
        if second_order:
            half = q1_gate(mixing_time / 2)
            for nid in range(n):
                em.apply_q1(half, nid)
        for (a, b), J in zip(energy.coupled_spin_pairs, energy.coupling_amplitudes):
            a, b = int(a), int(b)
            em.apply_q2(q2_gate(J, energy.fields[a] / deg[a], energy.fields[b] / deg[b], coupling_time), a, b)
        mix = q1_gate(mixing_time / 2 if second_order else mixing_time)
        for nid in range(n):
            em.apply_q1(mix, nid)
    rho = em.all_densities()
    order = [em._node_idx[i] for i in range(n)]
    config = None
    if sample_measurements:
        outcomes = [em.measure(nid, None if samples is None else float(samples[nid])) for nid in range(n)]
        config = 1 - 2 * np.array(outcomes, dtype=np.int64)
    return QuantumAnnealingResults(
        density_matrices=rho[order].cpu().numpy(),
        vidal_distances_after_regauging=em.after_regauging_vidal_distances.cpu().numpy(),
        truncation_affected_vidal_distances=em.truncated_affected_vidal_distances.cpu().numpy(),
        truncation_errors=np.array([float(x) for x in em.truncation_errors]),
        entropies=np.array([float(x) for x in em.entropies]),
        configuration=config,
    )


def eval_energy(energy: EnergyFunction, config: np.ndarray) -> float:
    """energy_evaluation.py:8-16: E(s) = -sum h s - sum J s_i s_j."""
    p = energy.coupled_spin_pairs
    return float(-(energy.fields @ config) - (config[p[:, 0]] * config[p[:, 1]]) @ energy.coupling_amplitudes)
