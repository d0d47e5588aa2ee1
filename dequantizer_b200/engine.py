"""Packed BP engine: the fast public path for a fixed graph and bond sizes.

Where the dict maps (``dequantizer_b200.maps``) pack and unpack Python dicts
on every call, ``BPEngine`` keeps node tensors and messages in device arenas
and exposes whole-graph operations on them:

* ``sweep()``            -- one BP sweep (mappings/belief_propagation.py:24-64)
  with the reference's synchronous or asynchronous (traversal-order)
  semantics, or a flooding schedule;
* ``distance()``         -- mean Frobenius distance between the last two
  message sets (mappings/messages_distance.py:14-22);
* ``run()``              -- sweeps to a tolerance, like the reference's
  driver loops (examples/3d_ising_canonicalization.py:137-145);
* ``vidal_gauge()`` / ``vidal_distance()`` / ``densities()``.

Host arrays can be loaded and read back through pinned staging buffers
(``load_tensors_host`` / ``read_messages_host``), the end-to-end path.
"""

from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .graph import TensorGraph
from .layout import GraphLayout
from .maps import Topology, bp_sweep, density_packed, vidal_distance_packed, vidal_gauge_packed

SCHEDULES = ("sync", "async", "flooding")


class BPEngine:
    def __init__(self, graph: TensorGraph, traversal: str = "dfs", schedule: str = "sync", device=None):
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {SCHEDULES}")
        if not torch.cuda.is_available():
            raise RuntimeError("BPEngine runs on the GPU only and no CUDA device is available")
        _lib.lib()
        self.graph = graph
        trav = list(graph.get_traversal_iterator(ordering=traversal))
        self.topo = Topology(trav, schedule == "sync", flooding=schedule == "flooding")
        chi = [e.dimension for e in self.topo.edges]
        self.layout = GraphLayout(self.topo.nodes, self.topo.edges, chi, device=device)
        L = self.layout
        self.T = L.new_tensor_arena()
        self.n2e = L.new_msg_arena()
        self.e2n = L.new_msg_arena()
        self._n2e_prev: Optional[torch.Tensor] = None
        self._e2n_prev: Optional[torch.Tensor] = None
        self._spare = (L.new_msg_arena(), L.new_msg_arena())
        self._partial = torch.empty(max(2 * L.n_halves, 1), dtype=torch.float64, device=L.device)
        nb = _lib.lib().dqz_bp_node_scratch_bytes(max(len(l) for l in self.topo.levels), L.max_slice(),
                                                 L.max_chi())
        self._scratch = torch.empty(nb, dtype=torch.uint8, device=L.device) if nb else None
        self._pinned = {}

    # -------------------------------------------------------------- load
    def load_tensors(self, tensors_by_node: Sequence) -> None:
        """Node tensors in traversal node order (numpy or torch, any complex dtype)."""
        L = self.layout
        for v, t in enumerate(tensors_by_node):
            tt = t if isinstance(t, torch.Tensor) else torch.from_numpy(np.asarray(t))
            o = int(L.node_off[v])
            self.T[o : o + tt.numel()] = tt.reshape(-1).to(L.device, torch.complex128)

    def load_messages(self, n2e_by_half: Sequence, e2n_by_half: Optional[Sequence] = None) -> None:
        L = self.layout
        for arena, mats in ((self.n2e, n2e_by_half), (self.e2n, e2n_by_half if e2n_by_half is not None else n2e_by_half)):
            for h, m in enumerate(mats):
                mm = m if isinstance(m, torch.Tensor) else torch.from_numpy(np.asarray(m))
                o = int(L.half_msg_off[h])
                arena[o : o + mm.numel()] = mm.reshape(-1).to(L.device, torch.complex128)

    def _pin(self, name, numel, dtype):
        buf = self._pinned.get(name)
        if buf is None or buf.numel() != numel or buf.dtype != dtype:
            buf = torch.empty(numel, dtype=dtype, pin_memory=True)
            self._pinned[name] = buf
        return buf

    def load_tensors_host(self, packed: torch.Tensor) -> None:
        """Asynchronous H2D of a packed host arena (complex64 or complex128,
        pinned) into the tensor arena, converted on the device."""
        if packed.dtype == torch.complex128:
            self.T.copy_(packed, non_blocking=True)
        else:
            stage = self._stage("t_stage", packed.numel(), packed.dtype)
            stage.copy_(packed, non_blocking=True)
            self.T.copy_(stage)

    def _stage(self, name, numel, dtype):
        buf = self._pinned.get("dev_" + name)
        if buf is None or buf.numel() != numel or buf.dtype != dtype:
            buf = torch.empty(numel, dtype=dtype, device=self.layout.device)
            self._pinned["dev_" + name] = buf
        return buf

    def load_messages_host(self, n2e: torch.Tensor, e2n: torch.Tensor) -> None:
        self.n2e.copy_(n2e, non_blocking=True)
        self.e2n.copy_(e2n, non_blocking=True)

    def read_messages_host(self, out_n2e: torch.Tensor) -> None:
        out_n2e.copy_(self.n2e, non_blocking=True)

    # ------------------------------------------------------------ compute
    def sweep(self, mid_event=None) -> None:
        """One BP sweep; the previous message set is kept for ``distance``.
        ``mid_event`` (a torch.cuda.Event) is recorded between the node
        updates and the edge pass, to time the node-update kernel alone."""
        n2e_new, e2n_new = self._spare
        L = self.layout
        src_sel, edge_new, levels = self.topo.device_tables(L.device)
        stream = _lib.stream_handle()
        ms, mc = L.max_slice(), L.max_chi()
        for halves in levels:
            _lib.call("dqz_bp_node_update", L.gptr, self.T.data_ptr(), self.n2e.data_ptr(), self.e2n.data_ptr(),
                      n2e_new.data_ptr(), src_sel.data_ptr(), halves.data_ptr(), halves.numel(), ms, mc,
                      _lib.ptr(self._scratch), stream)
        if mid_event is not None:
            mid_event.record(torch.cuda.current_stream())
        _lib.call("dqz_bp_edge_pass", L.gptr, self.n2e.data_ptr(), n2e_new.data_ptr(), edge_new.data_ptr(),
                  e2n_new.data_ptr(), mc, stream)
        self._spare = (self.n2e, self.e2n)
        self._n2e_prev, self._e2n_prev = self.n2e, self.e2n
        self.n2e, self.e2n = n2e_new, e2n_new

    def launches_per_sweep(self) -> int:
        return len(self.topo.levels) + 1

    def distance(self) -> torch.Tensor:
        """Mean Frobenius distance between the current and previous messages."""
        if self._n2e_prev is None:
            raise RuntimeError("distance() needs at least one sweep")
        L = self.layout
        out = torch.empty((), dtype=torch.float64, device=L.device)
        _lib.call("dqz_messages_distance", L.gptr, self.n2e.data_ptr(), self._n2e_prev.data_ptr(),
                  self.e2n.data_ptr(), self._e2n_prev.data_ptr(), self._partial.data_ptr(), out.data_ptr(),
                  L.max_chi(), _lib.stream_handle())
        return out

    def run(self, tol: float, max_sweeps: int = 1000, check_every: int = 1) -> int:
        """Sweeps until distance() <= tol (read back every ``check_every`` sweeps)."""
        for it in range(1, max_sweeps + 1):
            self.sweep()
            if it % check_every == 0 and float(self.distance()) <= tol:
                return it
        return max_sweeps

    def vidal_gauge(self, eps: float = 1e-10):
        return vidal_gauge_packed(self.layout, self.T, self.n2e, eps)

    def vidal_distance(self, G, lam, eps: float = 1e-10) -> torch.Tensor:
        return vidal_distance_packed(self.layout, G, lam, eps)

    def densities(self, nodes: Optional[List[int]] = None) -> torch.Tensor:
        nodes = list(range(self.layout.n_nodes)) if nodes is None else nodes
        return density_packed(self.layout, self.T, self.e2n, nodes)

    def messages(self) -> List[torch.Tensor]:
        return [self.layout.message_view(self.n2e, h) for h in range(self.layout.n_halves)]
