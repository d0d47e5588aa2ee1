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
* ``vidal_gauge()`` / ``vidal_distance()`` / ``densities()`` (FP64).

``precision="fp64"`` keeps complex128 arenas (the plain form);
``precision="fp32"`` keeps complex64 arenas and runs the sweeps in FP32
(degree-3 nodes with bonds of dimension 8 or 16), while the gauge,
distance and density computations are still done in FP64 on upcast copies.
Host arrays are loaded and read back through the ``*_host`` methods, the
end-to-end path.
"""

from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .graph import TensorGraph
from .layout import GraphLayout
from .maps import BF16_KERNELS, Topology, bp_sweep, density_packed, error_flag, vidal_distance_packed, vidal_gauge_packed

SCHEDULES = ("sync", "async", "flooding")
PRECISIONS = {"fp64": torch.complex128, "fp32": torch.complex64, "bf16": torch.complex64}


class BPEngine:
    def __init__(self, graph: TensorGraph, traversal: str = "dfs", schedule: str = "sync", precision: str = "fp64",
                 device=None, bf16_kernel: str = "tcgen05"):
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {SCHEDULES}")
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {tuple(PRECISIONS)}")
        if not torch.cuda.is_available():
            raise RuntimeError("BPEngine runs on the GPU only and no CUDA device is available")
        _lib.lib()
        self.graph = graph
        self.precision = precision
        self.dtype = PRECISIONS[precision]
        trav = list(graph.get_traversal_iterator(ordering=traversal))
        self.topo = Topology(trav, schedule == "sync", flooding=schedule == "flooding")
        chi = [e.dimension for e in self.topo.edges]
        self.layout = GraphLayout(self.topo.nodes, self.topo.edges, chi, device=device)
        L = self.layout
        if precision == "fp32" and not L.uniform_k3_chi():
            raise NotImplementedError("fp32 sweeps need degree-3 nodes with bonds of dimension 8 or 16")
        if precision == "bf16" and L.uniform_k3_chi() != 16:
            raise NotImplementedError("bf16 tensor-core sweeps need degree-3 nodes with bonds of dimension 16")
        self.T = self._arena(L.tensor_elems)
        self.n2e = self._arena(L.msg_elems)
        self.e2n = self._arena(L.msg_elems)
        self._prev = None
        self._spare = (self._arena(L.msg_elems), self._arena(L.msg_elems))
        self._partial = torch.empty(max(2 * L.n_halves, 1), dtype=torch.float64, device=L.device)
        self._stage = {}
        # bf16: node tensors also kept in BF16, rebuilt from T after every
        # load: the tcgen05 kernel's core layouts, or the mma_sync kernel's planes
        if bf16_kernel not in BF16_KERNELS:
            raise ValueError(f"bf16_kernel must be one of {tuple(BF16_KERNELS)}")
        self.bf16_kernel = bf16_kernel
        per_node = int(_lib.lib().dqz_bf16_umma_elems_per_node()) if bf16_kernel == "tcgen05" else 16384
        self.T_bf16 = (torch.empty(L.n_nodes * per_node, dtype=torch.bfloat16, device=L.device)
                       if precision == "bf16" else None)
        self._bf16_stale = True
        self._canon_graphs = {}  # canonicalise(): eps -> {message buffer at start -> (graph, outputs)}

    def _arena(self, n):
        return torch.zeros(max(n, 1), dtype=self.dtype, device=self.layout.device)

    @property
    def kernel(self) -> str:
        if self.precision == "bf16":
            return "bp_node_k3_umma" if self.bf16_kernel == "tcgen05" else "bp_node_k3_tc"
        return "bp_node_k3" if self.layout.uniform_k3_chi() else "bp_node_generic"

    # -------------------------------------------------------------- load
    def load_tensors(self, tensors_by_node: Sequence) -> None:
        """Node tensors in traversal node order (numpy or torch, any complex dtype)."""
        L = self.layout
        for v, t in enumerate(tensors_by_node):
            tt = t if isinstance(t, torch.Tensor) else torch.from_numpy(np.asarray(t))
            o = int(L.node_off[v])
            self.T[o : o + tt.numel()] = tt.reshape(-1).to(L.device, self.dtype)
        self._bf16_stale = True

    def load_messages(self, n2e_by_half: Sequence, e2n_by_half: Optional[Sequence] = None) -> None:
        L = self.layout
        e2n_by_half = e2n_by_half if e2n_by_half is not None else n2e_by_half
        for arena, mats in ((self.n2e, n2e_by_half), (self.e2n, e2n_by_half)):
            for h, m in enumerate(mats):
                mm = m if isinstance(m, torch.Tensor) else torch.from_numpy(np.asarray(m))
                o = int(L.half_msg_off[h])
                arena[o : o + mm.numel()] = mm.reshape(-1).to(L.device, self.dtype)

    def _staged(self, src: torch.Tensor, dst: torch.Tensor) -> None:
        """Asynchronous H2D of a pinned host arena into ``dst``; a dtype
        change happens on the device after the copy."""
        if src.dtype == dst.dtype:
            dst.copy_(src, non_blocking=True)
            return
        key = (src.numel(), src.dtype)
        buf = self._stage.get(key)
        if buf is None:
            buf = torch.empty(src.numel(), dtype=src.dtype, device=self.layout.device)
            self._stage[key] = buf
        buf.copy_(src, non_blocking=True)
        dst.copy_(buf)

    def load_tensors_host(self, packed: torch.Tensor) -> None:
        self._staged(packed, self.T)
        self._bf16_stale = True

    def load_messages_host(self, n2e: torch.Tensor, e2n: torch.Tensor) -> None:
        self._staged(n2e, self.n2e)
        self._staged(e2n, self.e2n)

    def read_messages_host(self, out_n2e: torch.Tensor) -> None:
        out_n2e.copy_(self.n2e, non_blocking=True)

    # ------------------------------------------------------------ compute
    def sweep(self, mid_event=None) -> None:
        """One BP sweep; the previous message set is kept for ``distance``.
        ``mid_event`` (a torch.cuda.Event) is recorded between the node
        updates and the edge pass, to time the node-update kernel alone."""
        n2e_new, e2n_new = self._spare
        if self.T_bf16 is not None and self._bf16_stale:
            pack = "dqz_pack_bf16_umma" if self.bf16_kernel == "tcgen05" else "dqz_pack_bf16_planes"
            _lib.call(pack, self.layout.gptr, self.T.data_ptr(), self.T_bf16.data_ptr(),
                      _lib.stream_handle())
            self._bf16_stale = False
        bp_sweep(self.layout, self.topo, self.T, self.n2e, self.e2n, n2e_new, e2n_new, mid_event,
                 T_bf16=self.T_bf16, bf16_kernel=self.bf16_kernel)
        self._spare = (self.n2e, self.e2n)
        self._prev = (self.n2e, self.e2n)
        self.n2e, self.e2n = n2e_new, e2n_new

    def launches_per_sweep(self) -> int:
        return len(self.topo.levels) + 1

    def check(self) -> None:
        """Raises when a kernel skipped a node of an unexpected shape."""
        if int(error_flag(self.layout.device).item()):
            raise RuntimeError("a BP kernel met a node outside its supported shape")

    def _c128(self, x: torch.Tensor) -> torch.Tensor:
        return x if x.dtype == torch.complex128 else x.to(torch.complex128)

    def distance(self) -> torch.Tensor:
        """Mean Frobenius distance between the current and previous messages (FP64)."""
        if self._prev is None:
            raise RuntimeError("distance() needs at least one sweep")
        L = self.layout
        out = torch.empty((), dtype=torch.float64, device=L.device)
        # keep the (possibly converted) operands alive across the call: a
        # temporary's memory could be handed to the next conversion otherwise
        ops = [self._c128(x) for x in (self.n2e, self._prev[0], self.e2n, self._prev[1])]
        _lib.call("dqz_messages_distance", L.gptr, *(x.data_ptr() for x in ops), self._partial.data_ptr(),
                  out.data_ptr(), L.max_chi(), _lib.stream_handle())
        return out

    def run(self, tol: float, max_sweeps: int = 1000, check_every: int = 1) -> int:
        """Sweeps until distance() <= tol (read back every ``check_every`` sweeps)."""
        for it in range(1, max_sweeps + 1):
            self.sweep()
            if it % check_every == 0 and float(self.distance()) <= tol:
                return it
        return max_sweeps

    def run_graphed(self, tol: float, max_sweeps: int = 1000, block: int = 8) -> int:
        """``run`` with every block of ``block`` sweeps and the distance that
        ends it captured once into a CUDA graph and replayed; the host reads
        the distance once per block. ``block`` must be even (message buffers
        rotate with period two, so each replay starts from the captured
        buffer assignment). Returns the number of sweeps done."""
        if block < 2 or block % 2:
            raise ValueError("block must be an even number >= 2")
        # two eager sweeps: allocations, kernel attributes and BF16 planes
        # happen before capture
        self.sweep()
        self.sweep()
        done = 2
        if float(self.distance()) <= tol or done >= max_sweeps:
            return done
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            for _ in range(block):
                self.sweep()
            dist = self.distance()
        self._graph = graph  # keep the graph (and its memory pool) alive with the engine
        while done < max_sweeps:
            graph.replay()
            done += block
            if float(dist) <= tol:
                break
        return done

    def _rotate(self) -> None:
        """The buffer reassignment of one sweep, without its kernels."""
        n2e_new, e2n_new = self._spare
        self._spare = (self.n2e, self.e2n)
        self._prev = (self.n2e, self.e2n)
        self.n2e, self.e2n = n2e_new, e2n_new

    def canonicalise(self, eps: float, max_iterations: int = 500, graphed: bool = True):
        """The canonicalisation loop of examples/3d_ising_canonicalization.py:137-145:
        repeat {one sweep, Vidal gauge, Vidal distance} until the distance is
        <= ``eps`` or ``max_iterations`` iterations; returns (distance of every
        iteration, Gamma arena, lambda arena) of the last iteration.

        With ``graphed``, iterations replay CUDA graphs of the whole iteration,
        one for each of the two message-buffer assignments the sweeps alternate
        between. They are captured after two eager iterations of the first call
        and kept with the engine (keyed by ``eps``), so later calls on new
        tensors or messages loaded into the same arenas replay from their first
        iteration. The host reads one scalar per iteration and the stopping rule
        is the eager one, so results equal the eager loop's bit for bit; the
        returned arenas are copies. BF16 engines run eagerly. Small
        graphs whose sweeps are many tiny level launches (asynchronous
        schedules) gain most."""
        graphed = graphed and self.T_bf16 is None  # BF16 node tensors are re-packed on the host side of a load
        cache = self._canon_graphs.setdefault(float(eps), {}) if graphed else {}
        hist = []
        G = lam = None
        vd = float("inf")

        def iteration():
            self.sweep()
            g_, l_ = self.vidal_gauge(eps)
            return g_, l_, self.vidal_distance(g_, l_, eps)

        while vd > eps and len(hist) < max_iterations:
            entry = cache.get(self.n2e.data_ptr())
            if entry is not None:
                graph, (G, lam, d) = entry
                graph.replay()
                self._rotate()
            elif graphed and len(hist) >= 2:
                # capturing records a sweep without running it: two captures
                # leave the buffer assignment where it was
                for _ in range(2):
                    start = self.n2e.data_ptr()
                    graph = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(graph):
                        out = iteration()
                    cache[start] = (graph, out)
                continue
            else:
                G, lam, d = iteration()
            vd = float(d)
            hist.append(vd)
        if cache:  # the last outputs may live in a graph's memory, which its next replay overwrites
            G, lam = G.clone(), lam.clone()
        return hist, G, lam

    def vidal_gauge(self, eps: float = 1e-10):
        return vidal_gauge_packed(self.layout, self._c128(self.T), self._c128(self.n2e), eps)

    def vidal_distance(self, G, lam, eps: float = 1e-10) -> torch.Tensor:
        return vidal_distance_packed(self.layout, G, lam, eps)

    def densities(self, nodes: Optional[List[int]] = None) -> torch.Tensor:
        nodes = list(range(self.layout.n_nodes)) if nodes is None else nodes
        return density_packed(self.layout, self._c128(self.T), self._c128(self.e2n), nodes)

    def messages(self) -> List[torch.Tensor]:
        return [self.layout.message_view(self.n2e, h) for h in range(self.layout.n_halves)]
