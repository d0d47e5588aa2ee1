"""Exact dense state-vector emulator on the GPU, the validation oracle of the
BP emulator (quantum_emulator/exact_quantum_emulator.py:11-147, same public
methods and qubit order: positions follow the nodes of the graph's default
traversal, position 0 is the most significant bit of the amplitude index).

The state is a complex128 vector of 2^n amplitudes in device memory (26
qubits = 1 GiB); every operation is a libdqz kernel (``dqz_sv_*``), one read
and one write of the state per gate. ``measure`` takes an optional uniform
sample like ``BPQuantumEmulator.measure``; without one it draws from a numpy
generator seeded by ``key`` (the reference draws from a JAX key).
"""

from typing import Dict, Optional

import numpy as np
import torch

from . import _lib
from .graph import Node, NodeID, TensorGraph


class DenseStateEmulator:
    def __init__(self, tensor_graph: TensorGraph, key: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("DenseStateEmulator runs on the GPU only")
        _lib.lib()
        self.n = tensor_graph.nodes_number
        if self.n < 1 or self.n > 34:
            raise NotImplementedError("the dense emulator covers 1..34 qubits")
        self.node2pos: Dict = {}
        pos = 0
        for element in tensor_graph.get_traversal_iterator() or iter([]):
            if isinstance(element, Node):
                self.node2pos[element.id] = pos
                pos += 1
        self.device = _lib.device()
        self.state = torch.empty(2**self.n, dtype=torch.complex128, device=self.device)
        self._rho = torch.empty(4, dtype=torch.complex128, device=self.device)
        nb = _lib.lib().dqz_sv_density_scratch_bytes(self.n)
        self._scratch = torch.empty(max(int(nb), 1), dtype=torch.uint8, device=self.device)
        self._rng = np.random.default_rng(key)
        self._set_basis(0)

    def _set_basis(self, index: int) -> None:
        _lib.call("dqz_sv_set_basis", self.state.data_ptr(), self.n, int(index), _lib.stream_handle())

    @staticmethod
    def _host_gate(gate, shape) -> np.ndarray:
        g = gate.detach().cpu().numpy() if isinstance(gate, torch.Tensor) else np.asarray(gate)
        g = np.ascontiguousarray(g, dtype=np.complex128)
        if g.shape != shape:
            raise ValueError(f"gate of shape {g.shape}, expected {shape}")
        return g

    def set_to_product_state(self, state: Dict[NodeID, int]) -> None:
        """exact_quantum_emulator.py:38-50."""
        shift = 0
        for node_id, pos in self.node2pos.items():
            if state[node_id] == 1:
                shift += 2 ** (self.n - pos - 1)
        self._set_basis(shift)

    def apply_q2(self, gate, controlling_node_id: NodeID, controlled_node_id: NodeID) -> None:
        """exact_quantum_emulator.py:60-80: gate (2, 2, 2, 2) = (o1, o2, i1, i2)."""
        g = self._host_gate(gate, (2, 2, 2, 2))
        _lib.call("dqz_sv_apply2", self.state.data_ptr(), self.n, self.node2pos[controlling_node_id],
                  self.node2pos[controlled_node_id], g.ctypes.data, _lib.stream_handle())

    def apply_q1(self, gate, node_id: NodeID) -> None:
        """exact_quantum_emulator.py:88-99: gate (2, 2) = (output, input)."""
        g = self._host_gate(gate, (2, 2))
        _lib.call("dqz_sv_apply1", self.state.data_ptr(), self.n, self.node2pos[node_id], g.ctypes.data,
                  _lib.stream_handle())

    def dens_q1(self, node_id: NodeID) -> torch.Tensor:
        """exact_quantum_emulator.py:107-121: 2 x 2 reduced density matrix."""
        _lib.call("dqz_sv_density1", self.state.data_ptr(), self.n, self.node2pos[node_id], self._rho.data_ptr(),
                  self._scratch.data_ptr(), _lib.stream_handle())
        return self._rho.clone().reshape(2, 2)

    def measure(self, node_id: NodeID, sample: Optional[float] = None) -> int:
        """exact_quantum_emulator.py:129-147: outcome 0 when rho_00 > sample,
        then projection and renormalisation."""
        p = float(self.dens_q1(node_id)[0, 0].real)
        u = float(self._rng.uniform()) if sample is None else float(sample)
        result, norm = (0, p) if p > u else (1, 1.0 - p)
        _lib.call("dqz_sv_project", self.state.data_ptr(), self.n, self.node2pos[node_id], result,
                  1.0 / np.sqrt(norm), _lib.stream_handle())
        return result
