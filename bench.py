"""Benchmark: BP edge-updates/s on a random 3-regular graph (1024 nodes,
bond dimension 16, physical dimension 2), one GPU per rank.

A step is one full BP sweep over every directed edge (3072 edge-updates) in
the reference's synchronous mode (one node-update launch + one edge pass).
``value`` is timed on the device with CUDA events per step, inputs resident
in HBM, L2 flushed (a 512 MB write) between steps outside the timed events.
``e2e`` is the same sweep through the public engine API with host buffers:
pinned complex64 node tensors and messages copied in, the sweep, the
node->edge messages copied back, all inside the timed region
(``BPEngine.sweep_host``: the copies stream in node ranges that are packed
and updated as they arrive, overlapping the transfers with the kernels).

``--impl reference`` times the CPU restatement of the reference algorithm
(numpy FP64 pass_through_node, one process per host core with one BLAS thread
each) on a bounded sample of the same workload.
With torchrun (N > 1) every rank runs an independent replica ("replicas
only": the sweep of one graph has no exchange step here).
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BP edge-updates/s & anneal steps/s vs plain FP64 on GPU at |Δ<Z>|≤1e-4"
UNIT = "edge-updates/s"
N_NODES, DEGREE, CHI, PHYS, SEED = 1024, 3, 16, 2, 0


def workload(rank: int = 0):
    """Graph, complex64 node tensors (node order of the DFS traversal) and
    PSD messages (half-edge order), seeded."""
    from dequantizer_b200.graph import get_random_regular_graph

    g = get_random_regular_graph(N_NODES, DEGREE, PHYS, CHI, SEED + rank)
    rng = np.random.default_rng(1000 + rank)
    size = CHI**DEGREE * PHYS
    scale = 1.0 / np.sqrt(2.0 * CHI**DEGREE)
    z = rng.standard_normal((N_NODES, size, 2), dtype=np.float32)
    tensors = ((z[..., 0] + 1j * z[..., 1]) * (scale / np.sqrt(2.0))).astype(np.complex64)
    a = rng.standard_normal((CHI, CHI, 2))
    a = a[..., 0] + 1j * a[..., 1]
    m = a @ a.conj().T
    m /= np.trace(m).real
    return g, tensors, m


def flops_per_edge_update(k=DEGREE, d=PHYS, chi=CHI):
    return 8 * k * d * chi ** (k + 1)


def bytes_per_edge_update(k=DEGREE, d=PHYS, chi=CHI, s=16):
    return s * (d * chi**k + 2 * k * chi * chi) / k


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def reduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


CPU_SAMPLE_NODES = 64  # node tensors each CPU worker cycles through (4 MB of complex64)


def _cpu_worker_init():
    from threadpoolctl import threadpool_limits

    threadpool_limits(1)  # one BLAS thread per worker process: the pool supplies the parallelism


def _cpu_worker(args):
    """One worker: the oracle's pass_through_node (complex128) over its share
    of the sampled node tensors for ``seconds``; returns (node updates, seconds)."""
    tensors, m, seconds, start = args
    from oracle import tensor_ops as OT

    shape = (CHI,) * DEGREE + (PHYS,)
    msgs = [m] * DEGREE
    t64 = [t.astype(np.complex128).reshape(shape) for t in tensors]
    done, i = 0, start
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        OT.pass_through_node(t64[i % len(t64)], msgs)
        done += 1
        i += 1
    return done, time.perf_counter() - t0


class CpuBaseline:
    """The oracle's pass_through_node on the host cores: ``procs`` worker
    processes (default: every core), started with spawn and limited to one
    BLAS thread each, every one cycling over the same sample of
    CPU_SAMPLE_NODES node tensors. The pool starts once; ``sample(seconds)``
    returns (edge-updates/s summed over the workers, workers, description)."""

    def __init__(self, tensors_c64, m, procs=None):
        import multiprocessing as mp

        self.procs = procs or os.cpu_count() or 1
        self.sample_t = np.ascontiguousarray(tensors_c64[:CPU_SAMPLE_NODES])
        self.m = m
        old = os.environ.get("OPENBLAS_NUM_THREADS")
        os.environ["OPENBLAS_NUM_THREADS"] = "1"
        try:
            self.pool = mp.get_context("spawn").Pool(self.procs, initializer=_cpu_worker_init)
        finally:
            if old is None:
                os.environ.pop("OPENBLAS_NUM_THREADS", None)
            else:
                os.environ["OPENBLAS_NUM_THREADS"] = old
        self.pool.map(_cpu_worker, [(self.sample_t[:2], m, 0.2, 0)] * self.procs)  # imports, untimed

    def sample(self, seconds):
        res = self.pool.map(_cpu_worker, [(self.sample_t, self.m, seconds, k) for k in range(self.procs)])
        rate = sum(DEGREE * n / dt for n, dt in res)
        nodes = sum(n for n, _ in res)
        return rate, self.procs, (f"{self.procs} processes x 1 BLAS thread, {nodes} nodes' pass_through_node "
                                  f"({DEGREE * nodes} edge-updates) in ~{seconds:.0f}s, cycling over "
                                  f"{len(self.sample_t)} of the workload's node tensors")

    @staticmethod
    def single(tensors_c64, m, seconds):
        with CpuBaseline(tensors_c64, m, procs=1) as one:
            return one.sample(seconds)

    def close(self):
        self.pool.close()
        self.pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _jax_note() -> str:
    """Whether the reference's own JAX CPU path could be timed on this host."""
    import importlib.util

    if importlib.util.find_spec("jax") is None:
        return "unavailable on this box (jax is not installed); the baseline is the numpy restatement"
    return "jax importable, but the reference package does not travel here; the baseline is the numpy restatement"


def run_reference(args, world, rank):
    if rank != 0:
        return
    g, tensors, m = workload(0)
    vals = []
    with CpuBaseline(tensors, m) as cpu:
        for _ in range(args.warmup):
            cpu.sample(0.5)
        for _ in range(args.steps):
            v, threads, sample = cpu.sample(args.ref_seconds)
            vals.append(v)
        single, _, _ = CpuBaseline.single(tensors, m, min(2.0, args.ref_seconds))
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 3 * N_NODES / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": "random 3-regular graph, 1024 nodes, chi=16, d=2: one synchronous BP sweep "
                   "(3072 edge-updates)", "sample_per_step": f"~{args.ref_seconds:.0f}s of node updates"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "numpy FP64 restatement of tensor_ops.pass_through_node, "
                                   + sample, "single_process_value": single},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_peak(torch, dtype):
    """cuBLAS GEMM throughput (best of 3, 8192^3) for a real dtype: the FP64
    (DGEMM) or FP32 (SGEMM, TF32 off) compute roofline of the node kernels."""
    n = 8192
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    return 2.0 * n**3 / best / 1e12


# DRAM bytes (read + write) per node-update launch from one ncu capture of
# the bench workload; profiles/ holds the summaries these come from.
NCU_TRAFFIC = {
    # dram__bytes_read.sum + dram__bytes_write.sum per launch, from the ncu
    # captures summarised under profiles/ (same workload: 1024-node 3-regular
    # graph, chi 16, one launch over all 3072 half-edges)
    ("bp_node_generic", "fp64"): 166.6e6,
    ("bp_node_k3", "fp64"): 158.0e6,
    ("bp_node_k3", "fp32"): 77.6e6,
    ("bp_node_k3_tc", "bf16"): 39.9e6,
    ("bp_node_k3_umma", "bf16"): 75.0e6,
}


def time_engine(args, world, g, packed_c64, m, precision, flush, clk=None):
    """Device-timed sweeps and end-to-end sweeps for one precision."""
    import torch

    from dequantizer_b200.engine import BPEngine

    eng = BPEngine(g, traversal="dfs", schedule="sync", precision=precision)
    L = eng.layout
    mdt = torch.complex128 if precision == "fp64" else torch.complex64
    n2e_host = torch.from_numpy(np.tile(m.reshape(-1), L.n_halves)).to(mdt).pin_memory()
    e2n_host = n2e_host.clone().pin_memory()
    out_host = torch.empty_like(n2e_host).pin_memory()
    eng.load_tensors_host(packed_c64)
    eng.load_messages_host(n2e_host, e2n_host)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        eng.sweep()
    torch.cuda.synchronize()
    barrier(world)
    times, node_times = [], []
    for _ in range(args.steps):
        flush.zero_()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        eng.sweep(mid_event=e1)
        e2.record(stream)
        e2.synchronize()
        times.append(e0.elapsed_time(e2) * 1e-3)
        node_times.append(e0.elapsed_time(e1) * 1e-3)
    barrier(world)
    e_times = []
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        eng.sweep_host(packed_c64, n2e_host, e2n_host, out_host, chunks=args.e2e_chunks)
        e.record(stream)
        e.synchronize()
        e_times.append(s.elapsed_time(e) * 1e-3)
    eng.check()
    edge_updates = L.n_halves
    total = reduce_max(sum(times), world)
    e_total = reduce_max(sum(e_times), world)
    h2d = packed_c64.numel() * packed_c64.element_size() + 2 * n2e_host.numel() * n2e_host.element_size()
    return {
        "value": world * edge_updates * args.steps / total,
        "ms_per_step": total / args.steps * 1e3,
        "node_ms": float(np.mean(node_times)) * 1e3,
        "e2e": world * edge_updates * args.steps / e_total,
        "h2d": h2d,
        "d2h": out_host.numel() * out_host.element_size(),
        "launches": eng.launches_per_sweep() * args.steps,
        "kernel": eng.kernel,
        "edge_updates": edge_updates,
    }


def packed_inputs(g, tensors):
    """Node tensors in the engine's node order (DFS traversal), flattened."""
    import torch

    from dequantizer_b200.maps import Topology

    topo = Topology(list(g.get_traversal_iterator(ordering="dfs")), True)
    pos = {nid: i for i, nid in enumerate(g.nodes.keys())}
    perm = np.array([pos[n.id] for n in topo.nodes])
    return torch.from_numpy(np.ascontiguousarray(tensors[perm]).reshape(-1)).pin_memory()


def convergence_study(seeds=(0, 1, 2), tol=1e-6, max_sweeps=400, bf16_tol=1e-4, bf16_max_sweeps=60):
    """BP run to a message distance of ``tol`` from the same start in each
    form, then the Vidal gauge and the one-site densities (all FP64 on the
    final messages), for several seeds of the bench workload:
    * fp64: FP64 sweeps to ``tol``;
    * fp32: FP32 sweeps to ``tol``;
    * mixed: BF16 tensor-core sweeps to ``bf16_tol`` (above their rounding
      floor of ~5e-5; the distance read every second sweep, at most
      ``bf16_max_sweeps``), then an FP32 refinement tail to ``tol``.
    Per form: sweeps, device time to the tolerance (CUDA events around the
    loop, distance read back every sweep), and against FP64 the largest
    |delta lambda| over all bond spectra, the largest |delta rho_i| entry over
    all one-site densities and the largest |delta <Z_i>|."""
    import torch

    from dequantizer_b200.engine import BPEngine

    def engine(g, prec, packed, m):
        eng = BPEngine(g, traversal="dfs", schedule="sync", precision=prec)
        mdt = torch.complex128 if prec == "fp64" else torch.complex64
        msgs = torch.from_numpy(np.tile(m.reshape(-1), eng.layout.n_halves)).to(mdt)
        eng.load_tensors_host(packed)
        eng.load_messages_host(msgs, msgs)
        return eng

    def timed(fn):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        out = fn()
        e.record()
        e.synchronize()
        return out, s.elapsed_time(e)

    def observables(eng):
        _, lam = eng.vidal_gauge(1e-10)
        rho = eng.densities()
        z = (rho[:, 0, 0] - rho[:, 1, 1]).real
        return lam, rho, z

    per_seed = []
    for seed in seeds:
        g, tensors, m = workload(seed)
        packed = packed_inputs(g, tensors)
        res = {}
        e64 = engine(g, "fp64", packed, m)
        n64, t64 = timed(lambda: e64.run(tol, max_sweeps))
        ref = observables(e64)
        res["fp64"] = {"sweeps": n64, "ms": t64, "final_distance": float(e64.distance())}
        e32 = engine(g, "fp32", packed, m)
        n32, t32 = timed(lambda: e32.run(tol, max_sweeps))
        res["fp32"] = {"sweeps": n32, "ms": t32, "final_distance": float(e32.distance()), "obs": observables(e32)}
        ebf = engine(g, "bf16", packed, m)
        ebf.sweep()  # BF16 layouts packed and kernel attributes set outside the timed loop
        ebf.load_messages_host(torch.from_numpy(np.tile(m.reshape(-1), ebf.layout.n_halves)).to(torch.complex64),
                               torch.from_numpy(np.tile(m.reshape(-1), ebf.layout.n_halves)).to(torch.complex64))
        etail = engine(g, "fp32", packed, m)

        def mixed():
            nb = ebf.run(bf16_tol, bf16_max_sweeps, check_every=2)
            etail.n2e.copy_(ebf.n2e)
            etail.e2n.copy_(ebf.e2n)
            nt = etail.run(tol, max_sweeps)
            return nb, nt

        (nb, nt), tm = timed(mixed)
        res["mixed"] = {"sweeps_bf16": nb, "sweeps_fp32_tail": nt, "ms": tm,
                        "final_distance": float(etail.distance()), "obs": observables(etail)}
        for k in ("fp32", "mixed"):
            lam, rho, z = res[k].pop("obs")
            res[k]["max_abs_dlambda"] = float((lam - ref[0]).abs().max())
            res[k]["max_abs_drho"] = float((rho - ref[1]).abs().max())
            res[k]["max_abs_dZ"] = float((z - ref[2]).abs().max())
        per_seed.append(res)
    worst = lambda k, q: max(r[k][q] for r in per_seed)  # noqa: E731
    mean = lambda k, q: float(np.mean([r[k][q] for r in per_seed]))  # noqa: E731
    out = {"tol": tol, "bf16_handover_tol": bf16_tol, "seeds": list(seeds), "bound_dZ": 1e-4,
           "per_seed": per_seed}
    for k in ("fp32", "mixed"):
        out[k] = {q: worst(k, q) for q in ("max_abs_dlambda", "max_abs_drho", "max_abs_dZ")}
        out[k]["ok"] = out[k]["max_abs_dZ"] <= 1e-4
    for k in ("fp64", "fp32", "mixed"):
        out.setdefault(k, {})["mean_ms_to_tol"] = mean(k, "ms")
    out["time_to_tol_speedup_mixed_vs_fp64"] = out["fp64"]["mean_ms_to_tol"] / out["mixed"]["mean_ms_to_tol"]
    out["time_to_tol_speedup_fp32_vs_fp64"] = out["fp64"]["mean_ms_to_tol"] / out["fp32"]["mean_ms_to_tol"]
    return out


def bf16_sweep_accuracy(g, packed_c64, m, sweeps):
    """The per-sweep claim: the same number of BF16 tensor-core sweeps as FP64
    needs for the tolerance, from the same start; max |delta <Z_i>| against FP64."""
    import torch

    from dequantizer_b200.engine import BPEngine

    z = {}
    for prec in ("fp64", "bf16"):
        eng = BPEngine(g, traversal="dfs", schedule="sync", precision=prec)
        mdt = torch.complex128 if prec == "fp64" else torch.complex64
        msgs = torch.from_numpy(np.tile(m.reshape(-1), eng.layout.n_halves)).to(mdt)
        eng.load_tensors_host(packed_c64)
        eng.load_messages_host(msgs, msgs)
        for _ in range(sweeps):
            eng.sweep()
        rho = eng.densities()
        z[prec] = (rho[:, 0, 0] - rho[:, 1, 1]).real
    return float((z["bf16"] - z["fp64"]).abs().max())


def _events_time(fn):
    """(result, seconds) of fn() between CUDA events on the current stream."""
    import torch

    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    out = fn()
    e.record()
    e.synchronize()
    return out, s.elapsed_time(e) * 1e-3


def workload_suite(args):
    """Bounded runs of the other workloads, reported as extra keys of the
    default line (each names its sample; none is the headline):
    * ising3d -- the 3-D Ising canonicalisation in full (6x6x6 open lattice,
      chi 2, five betas, Vidal distance <= 1e-10; asynchronous DFS sweeps, one
      cooperative launch each), BP iterations/s, and the oracle's iteration
      (numpy, one core) timed on a few iterations of the same loop;
    * anneal -- 64 instances (n ~ U{100..1000} even, J = +-1), chi 16,
      second-order steps at s = 0.5 from the |+> state (warm-up steps first, so
      every bond is at 16), FP64 and mixed precision, instance-steps/s;
      the densities of both forms after the timed steps compared;
    * eagle -- the 127-qubit kicked-Ising run's first Trotter steps (bonds
      growing towards 32), Trotter steps/s;
    * grad -- the annealing-schedule gradient's first Trotter steps (512-node
      3-regular graph, J = +-1, chi 16, dt 0.1, s_t = (t + 1/2) / 200,
      checkpoints every 10): forward and gradient seconds."""
    import torch

    from dequantizer_b200.annealing import BatchedAnnealer
    from dequantizer_b200.workloads import ising_sqrt_partition, random_regular_energy, run_eagle_simulation

    out = {}
    # ---- 3-D Ising canonicalisation (config 1)
    betas = [0.1, 0.2, 0.3, 0.4, 0.5]
    kw = dict(lattice_sizes=[6, 6, 6], betas=betas, coupling=-1.0, field_strength=0.5, accuracy=1e-10,
              open_boundary=True, synchronous_update=False, key=42, traversal_type="dfs", max_iterations=500)
    ising_sqrt_partition(**kw)
    res, dt = _events_time(lambda: ising_sqrt_partition(**kw))
    iters = int(sum(res.number_of_iterations))
    out["ising3d"] = {"unit": "BP iterations/s", "value": iters / dt, "iterations_per_scan": iters, "scan_s": dt,
                      "average_magnetization": [float(x) for x in res.average_magnetization],
                      "cpu_oracle_iterations_per_s": _ising_oracle_rate(), "cpu_cores": 1}
    # ---- batched annealing, 64 instances, chi 16, mid-schedule (config 4)
    rng = np.random.default_rng(0)
    sizes = [int(2 * rng.integers(50, 501)) for _ in range(64)]
    energies = [random_regular_energy(n, 3, seed=1000 + i) for i, n in enumerate(sizes)]
    dt_step, s_mid, dt_warm = 0.1, 0.5, args.suite_anneal_warm_dt
    anneal = {"instances": 64, "nodes": int(sum(sizes)), "chi": 16, "s": s_mid, "dt": dt_step,
              "warmup_steps": args.suite_anneal_warmup, "timed_steps": args.suite_anneal_steps,
              "warmup_dt": dt_warm,
              "sample": "second-order steps (dt 0.1) at s = 0.5 from the |+> state after warm-up steps of a larger dt "
                        "that entangle the state (every bond at 16, regauges that sweep), not the annealed trajectory"}
    rho = {}
    for prec in ("fp64", "mixed"):
        ba = BatchedAnnealer(energies, max_chi=16, accuracy=1e-5, max_belief_propagation_iterations=100,
                             precision=prec)
        for i in range(args.suite_anneal_warmup):
            ba.step(-dt_warm * (1 - s_mid), dt_warm * s_mid, first=(i == 0), second_order=True)
        n0, b0 = len(ba.bp_iterations), len(ba.bf16_sweeps)

        def steps():
            for _ in range(args.suite_anneal_steps):
                ba.step(-dt_step * (1 - s_mid), dt_step * s_mid, first=False, second_order=True)

        _, dt = _events_time(steps)
        rho[prec] = ba.densities()
        anneal[prec] = {"unit": "instance-steps/s", "value": 64 * args.suite_anneal_steps / dt,
                        "ms_per_step": dt / args.suite_anneal_steps * 1e3,
                        "uniform_bond_16": bool(ba.layout.uniform_k3_chi() == 16),
                        "fp64_sweeps_per_regauge": float(np.mean(ba.bp_iterations[n0:])),
                        "bf16_sweeps_per_regauge": (float(np.mean(ba.bf16_sweeps[b0:])) if ba.bf16_sweeps[b0:]
                                                    else 0.0),
                        "fp32_sweeps_per_regauge": (float(np.mean(ba.fp32_sweeps[b0:])) if ba.fp32_sweeps[b0:]
                                                    else 0.0),
                        "gauge_evaluations_per_regauge": float(np.mean(ba.vd_checks[n0:]))}
        del ba
        torch.cuda.empty_cache()
    anneal["mixed_over_fp64"] = anneal["mixed"]["value"] / anneal["fp64"]["value"]
    dz = max(float(np.abs((a[:, 0, 0] - a[:, 1, 1]).real - (b[:, 0, 0] - b[:, 1, 1]).real).max())
             for a, b in zip(rho["mixed"], rho["fp64"]))
    anneal["max_abs_dZ_mixed_vs_fp64"] = dz
    out["anneal"] = anneal
    # ---- kicked Ising on the 127-qubit heavy-hex lattice (config 3), first steps
    n_eagle = args.suite_eagle_steps
    (z, em), dt = _events_time(lambda: run_eagle_simulation(
        max_chi=32, layers_per_regauging=1, trotter_steps=n_eagle, accuracy=1e-5, theta=0.6, is_infinite=False,
        colour_classes=True, all_qubits=True))
    out["eagle"] = {"unit": "Trotter steps/s", "value": n_eagle / dt, "steps": n_eagle,
                    "max_bond": int(em._layout.edge_chi.max()),
                    "sample": f"the first {n_eagle} of the 20 steps (bonds growing towards 32)"}
    del em
    torch.cuda.empty_cache()
    # ---- annealing-schedule gradient (config 5), first steps
    n_grad = args.suite_grad_steps
    if n_grad > 0:
        from dequantizer_b200.anneal_grad import AnnealingGradient

        try:
            ag = AnnealingGradient(random_regular_energy(512, 3, seed=500, field_std=0.0), max_chi=16, dt=0.1,
                                   checkpoint_every=10, bp_tol=1e-12)
            s_sched = (np.arange(n_grad) + 0.5) / 200
            E_fwd, t_fwd = _events_time(lambda: ag.energy_value(s_sched))
            (E, grad), t_grad = _events_time(lambda: ag.value_and_grad(s_sched))
            out["grad"] = {"unit": "s", "forward_s": t_fwd, "gradient_s": t_grad,
                           "gradient_over_forward": t_grad / t_fwd, "steps": n_grad,
                           "energy_matches_forward": abs(E - E_fwd) < 1e-12 * max(1.0, abs(E)),
                           "grad_norm": float(np.linalg.norm(grad)),
                           "sample": f"the first {n_grad} of the 200 steps (dt 0.1, s_t = (t + 1/2) / 200), "
                                     "512 nodes, chi 16, checkpoints every 10"}
        except Exception as exc:  # reported, not raised: the headline line still prints
            out["grad"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def _ising_oracle_rate(iterations=3):
    """The oracle's canonicalisation iteration (asynchronous DFS sweep, Vidal
    gauge, Vidal distance; numpy FP64, one process) on the 6x6x6 lattice at
    beta = 0.3: iterations/s over a few iterations."""
    from dequantizer_b200.graph import get_nd_lattice
    from dequantizer_b200.initializers import get_message_random_nonnegative_initializer, get_potts_initializer
    from oracle import maps as OM

    lat = get_nd_lattice([6, 6, 6], 2, 2, True)
    trav = list(lat.get_traversal_iterator(ordering="dfs"))
    bp, vg, vd = (OM.get_belief_propagation_map(trav), OM.get_vidal_gauge_fixing_map(trav, 1e-10),
                  OM.get_vidal_gauge_distance_map(trav, 1e-10))
    spins = np.array([1.0, -1.0])
    init = get_potts_initializer(np.exp(0.3 * np.tensordot(spins, spins, axes=0)), np.exp(-0.15 * spins))
    tensors = OM.init_tensors(lat, init)
    msgs = lat.init_messages(get_message_random_nonnegative_initializer(42))
    t0 = time.perf_counter()
    for _ in range(iterations):
        msgs = bp(tensors, msgs)
        t, lam = vg(tensors, msgs)
        vd(t, lam)
    return iterations / (time.perf_counter() - t0)


def run_ours(args, world, rank, local):
    import torch

    g, tensors, m = workload(rank)
    packed_c64 = packed_inputs(g, tensors)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    precs = [args.only] if args.only else ["fp64", "fp32", "bf16"]
    res = {}
    with ClockSampler(local) as clk:
        for p in precs:
            res[p] = time_engine(args, world, g, packed_c64, m, p, flush)
    if args.only:
        r = res[args.only]
        if rank == 0:
            print(json.dumps({"only": args.only, "value": r["value"], "node_ms": r["node_ms"],
                              "kernel": r["kernel"], "e2e": r["e2e"]}), flush=True)
        return
    acc = None
    if not args.no_accuracy:
        acc = convergence_study()
        acc["bf16_same_sweeps_max_abs_dZ"] = bf16_sweep_accuracy(g, packed_c64, m,
                                                                  acc["per_seed"][0]["fp64"]["sweeps"])
    peaks = {}
    if rank == 0:
        peaks["fp64"] = measure_peak(torch, torch.float64)
        peaks["fp32"] = measure_peak(torch, torch.float32)
    if rank != 0:
        return
    r64, r32, rbf = res["fp64"], res["fp32"], res["bf16"]
    fl = flops_per_edge_update() * rbf["edge_updates"]
    mp = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mp = json.load(f)
    except OSError:
        pass

    def roof(r, prec):
        ach = fl / (r["node_ms"] * 1e-3) / 1e12
        if prec == "bf16":
            peak = mp.get("bf16_tflops") or 1590.0
            src = "bf16_tflops of MEASURED_PEAKS.json (cuBLAS bf16 burst)" if mp.get("bf16_tflops") else \
                "fallback 1.59 PFLOP/s"
        else:
            peak = peaks[prec]
            src = ("cuBLAS DGEMM" if prec == "fp64" else "cuBLAS SGEMM (TF32 off)") + \
                " 8192^3 measured in this run (not in MEASURED_PEAKS.json)"
        return {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                "frac": ach / peak if peak else None,
                "traffic": NCU_TRAFFIC.get((r["kernel"], prec)),
                "kernel": r["kernel"], "peak_source": src,
                "flops_per_launch": fl, "launch_ms": r["node_ms"],
                "algorithmic_bytes_per_launch": r["edge_updates"] * bytes_per_edge_update(
                    s=16 if prec == "fp64" else 8)}

    cpu_v, cores, sample, cpu1 = (None, None, None, None)
    if world == 1 and not args.no_cpu:
        with CpuBaseline(tensors, m) as cpu:
            cpu_v, cores, sample = cpu.sample(args.cpu_seconds)
        # one worker process with one BLAS thread: the single-core figure
        cpu1, _, _ = CpuBaseline.single(tensors, m, min(4.0, args.cpu_seconds))
    suite = None
    if world == 1 and not args.no_suite:
        try:
            suite = workload_suite(args)
        except Exception as exc:  # an auxiliary block: report it, keep the headline line
            suite = {"error": f"{type(exc).__name__}: {exc}"}
    line = {
        "metric": METRIC, "value": rbf["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": rbf["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 tensor-core products, fp32 accumulate (c64 storage)",
        "data": "synthetic",
        "config": {
            "workload": "random 3-regular graph (pairing model, seed 0), 1024 nodes, chi=16, d=2, complex64 "
                        "node tensors: one synchronous BP sweep = 3072 edge-updates per step",
            "precision": "mixed: BF16 tensor-core contractions with FP32 accumulation and per-sweep trace "
                         "normalisation; eigen/SVD gauge, distance and densities in FP64",
            "schedule": "reference synchronous sweep",
            "l2": "flushed between steps (512 MB write)", "parallelism": f"replicas x{world}",
        },
        "fp64": {"value": r64["value"], "ms_per_step": r64["ms_per_step"], "e2e": r64["e2e"],
                 "roofline": roof(r64, "fp64")},
        "fp32": {"value": r32["value"], "ms_per_step": r32["ms_per_step"], "e2e": r32["e2e"],
                 "roofline": roof(r32, "fp32")},
        "speedup_vs_fp64": rbf["value"] / r64["value"],
        "accuracy": acc,
        "roofline": roof(rbf, "bf16"),
        "cpu_baseline": {"value": cpu_v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                         "single_process_value": cpu1, "reference_jax_cpu": _jax_note()},
        "e2e": {"value": rbf["e2e"], "unit": UNIT, "h2d_bytes_per_step": rbf["h2d"],
                "d2h_bytes_per_step": rbf["d2h"]},
        "gpu_launches": rbf["launches"],
        "clocks": clk.summary(),
        "other_workloads": suite,
    }
    print(json.dumps(line), flush=True)


def profile_hook(spec):
    """``--profile-steps A:B`` -> a callable(step) that opens the CUDA
    profiler range before step A and closes it before step B (for
    ``ncu --profile-from-start off`` captures of a few steps); None without."""
    if not spec:
        return None
    import torch

    a, b = (int(x) for x in spec.split(":"))

    def hook(step):
        if step == a:
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStart()
        elif step == b:
            torch.cuda.synchronize()
            torch.cuda.cudart().cudaProfilerStop()

    return hook


def run_anneal(args, world, rank, local):
    """Batched annealing: ``--instances`` random 3-regular instances with n
    uniform in [100, 1000] (even), J = +-1, h = 0, all advanced together by
    second-order Trotter steps of H(s) = -(1-s) sum X + s sum J ZZ with
    dt = total_time / n_steps (reference gate forms with tau_mix = -dt (1 - s),
    tau_coupling = dt s). A step is one Trotter step of every instance
    (regauge to the BP accuracy, all two-site gates, mixing); the unit is
    instance-steps/s. Instances are sharded over ranks (replicas)."""
    import torch

    from dequantizer_b200.annealing import BatchedAnnealer
    from dequantizer_b200.replicas import shard_weighted
    from dequantizer_b200.workloads import random_regular_energy

    rng = np.random.default_rng(0)
    sizes = [int(2 * rng.integers(50, 501)) for _ in range(args.instances)]
    mine = shard_weighted(sizes, world, rank)
    energies = [random_regular_energy(sizes[i], 3, seed=1000 + i) for i in mine]
    n_steps = args.trotter_steps
    dt = 20.0 / n_steps
    s_of = [t / (n_steps - 1) for t in range(n_steps)]
    ba = BatchedAnnealer(energies, max_chi=args.chi, accuracy=1e-5, max_belief_propagation_iterations=100,
                         precision=args.anneal_precision)
    if args.anneal_sample == "mid":
        # the suite's sample: warm-up steps of a larger dt at s = 0.5 entangle
        # the state (every bond at the cap), then steps of dt at s = 0.5
        s_of = [0.5] * n_steps
    torch.cuda.synchronize()
    t = 0
    for _ in range(args.warmup):
        s = s_of[t % n_steps]
        dw = args.suite_anneal_warm_dt if args.anneal_sample == "mid" else dt
        ba.step(-dw * (1 - s), dw * s, first=(t == 0), second_order=True)
        t += 1
    torch.cuda.synchronize()
    barrier(world)
    sw0, bf0 = len(ba.bp_iterations), len(ba.bf16_sweeps)
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        hook = profile_hook(args.profile_steps)
        for i in range(args.steps):
            if hook:
                hook(i)
            s = s_of[t % n_steps]
            ba.step(-dt * (1 - s), dt * s, first=False, second_order=True)
            t += 1
        if hook:
            hook(args.steps)
        e1.record()
        e1.synchronize()
    elapsed = reduce_max(e0.elapsed_time(e1) * 1e-3, world)
    # edge-updates inside the timed regauges: per sweep, every half-edge of the active instances
    halves = np.array([ba.half_range[k][1] - ba.half_range[k][0] for k in range(ba.n_inst)])
    upd = sum(int(np.dot(np.array(it), halves)) for it in ba.bp_iterations[sw0:])
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "batched annealing", "value": world * len(energies) * args.steps / elapsed,
            "unit": "instance-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "dtype": "c128" if args.anneal_precision == "fp64" else "bf16 + fp32 regauge sweeps + c128",
            "data": "synthetic",
            "config": {"instances": args.instances, "nodes": int(sum(sizes)), "chi": args.chi,
                       "trotter_steps": n_steps, "dt": dt, "order": 2, "bp_accuracy": 1e-5,
                       "bp_schedule": "synchronous, per-instance convergence"},
            "timed_s_range": [s_of[args.warmup % n_steps], s_of[(t - 1) % n_steps]],
            "sample": args.anneal_sample,
            "bp_edge_updates_per_s_rank0": upd / elapsed,
            "bp_sweeps_per_regauge_rank0": {"mean": float(np.mean(ba.bp_iterations[sw0:])),
                                            "max": int(np.max(ba.bp_iterations[sw0:]))},
            "precision": args.anneal_precision,
            "bf16_sweeps_per_regauge_rank0": (float(np.mean(ba.bf16_sweeps[bf0:])) if ba.bf16_sweeps[bf0:]
                                              else None),
            "fp32_sweeps_per_regauge_rank0": (float(np.mean(ba.fp32_sweeps[bf0:])) if ba.fp32_sweeps[bf0:]
                                              else None),
            "clocks": clk.summary(),
        }), flush=True)


def run_grad(args, world, rank, local):
    """Gradient of the final annealing energy E = sum J <ZZ> with respect to
    the per-step schedule values s_t: a random 3-regular graph of
    ``--grad-nodes`` nodes (default 512) with J = +-1, h = 0, chi = ``--chi``,
    ``--trotter-steps`` second-order steps (dt = 20 / steps), s_t initialised
    linear at the step midpoints, s_t = (t + 1/2) / N (a coupling step with
    s_t = 0 exactly is the identity, where the canonical form is not
    differentiable), checkpoints every 10 steps. A step of this workload is one full
    gradient (forward + checkpointed reverse pass); the unit is s/gradient.
    The gradient is checked against central finite differences along one
    random schedule direction, h = 1e-4 and 1e-5 (the truncated map has
    near-kinks where singular values at the truncation cut nearly cross, so the
    h = 1e-4 difference is not converged at this size). Each rank
    differentiates its own instance (replicas)."""
    import torch

    from dequantizer_b200.anneal_grad import AnnealingGradient
    from dequantizer_b200.workloads import random_regular_energy

    n_steps = args.trotter_steps
    energy = random_regular_energy(args.grad_nodes, 3, seed=500 + rank, field_std=0.0)
    ag = AnnealingGradient(energy, max_chi=args.chi, dt=20.0 / n_steps, checkpoint_every=10, bp_tol=1e-12)
    s = (np.arange(n_steps) + 0.5) / n_steps
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E_fwd = ag.energy_value(s)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    barrier(world)
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        E, grad = ag.value_and_grad(s)
        e1.record()
        e1.synchronize()
    elapsed = reduce_max(e0.elapsed_time(e1) * 1e-3, world)
    fd_info = None
    if not args.no_accuracy:
        d = np.random.default_rng(1).standard_normal(n_steps)
        ad = float(grad @ d)
        fd_info = {"directional_adjoint": ad, "target_rel_err": 1e-5}
        for h in (1e-4, 1e-5):
            fd = (ag.energy_value(s + h * d) - ag.energy_value(s - h * d)) / (2 * h)
            fd_info["fd_h%.0e" % h] = fd
            fd_info["rel_err_h%.0e" % h] = abs(ad - fd) / max(abs(fd), 1e-12)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "annealing-schedule gradient", "value": elapsed, "unit": "s/gradient",
            "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": elapsed * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"nodes": args.grad_nodes, "degree": 3, "couplings": "+-1", "chi": args.chi,
                       "trotter_steps": n_steps, "dt": 20.0 / n_steps, "order": 2, "checkpoint_every": 10,
                       "schedule": "s_t = (t + 1/2) / N",
                       "bp": "flooding sweeps to max change 1e-12 (fixed point)"},
            "energy": E, "forward_s": t_fwd, "gradient_over_forward": elapsed / t_fwd,
            "grad_norm": float(np.linalg.norm(grad)), "finite_difference_check": fd_info,
            "forward_energy_matches": abs(E - E_fwd) < 1e-12 * max(1.0, abs(E)),
            "clocks": clk.summary(),
        }), flush=True)


def run_ising3d(args, world, rank, local):
    """3-D Ising square-root network (examples/3d_ising_canonicalization.py:89-160):
    6 x 6 x 6 open lattice, bond dimension 2, Potts tensors with J = -1 and field
    h = 0.5 at beta = 0.1 ... 0.5; for each beta, asynchronous DFS sweeps from the
    seeded non-negative messages, each followed by the Vidal gauge and the Vidal
    distance, until that distance is <= 1e-10 (at most 500 sweeps). A step is one
    scan over the five betas; the unit is BP iterations/s (sweep + gauge +
    distance). Work is tiny (7.6 MFLOP per sweep) and launch / latency bound, so
    no roofline fraction is reported. Ranks run replicas."""
    import torch

    from dequantizer_b200.workloads import ising_sqrt_partition

    betas = [0.1, 0.2, 0.3, 0.4, 0.5]
    kw = dict(lattice_sizes=[6, 6, 6], betas=betas, coupling=-1.0, field_strength=0.5, accuracy=1e-10,
              open_boundary=True, synchronous_update=False, key=42, traversal_type="dfs", max_iterations=500)
    for _ in range(args.warmup):
        ising_sqrt_partition(**kw)
    torch.cuda.synchronize()
    barrier(world)
    iters = 0
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            res = ising_sqrt_partition(**kw)
            iters += sum(res.number_of_iterations)
        e1.record()
        e1.synchronize()
    elapsed = reduce_max(e0.elapsed_time(e1) * 1e-3, world)
    n_edges = 3 * 6 * 6 * 5
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "3-D Ising canonicalisation", "value": world * iters / elapsed,
            "unit": "BP iterations/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"lattice": "6x6x6 open", "chi": 2, "d": 2, "coupling": -1.0, "field": 0.5,
                       "betas": betas, "vidal_distance_tol": 1e-10, "max_sweeps": 500,
                       "schedule": "asynchronous DFS sweep + Vidal gauge + Vidal distance per iteration"},
            "iterations_per_scan": iters // max(args.steps, 1),
            "edge_updates_per_s": world * iters * 2 * n_edges / elapsed,
            "average_magnetization": res.average_magnetization, "roofline": None,
            "clocks": clk.summary(),
        }), flush=True)


def run_eagle(args, world, rank, local):
    """Kicked Ising on the 127-qubit heavy-hex lattice (examples/ibm_eagle_processor.py:56-145):
    RX(0.6) on every qubit and RZZ(-pi/2) on every edge per Trotter step, the
    RZZ gates in the three classes of a proper edge colouring with a Vidal
    regauge (BP accuracy 1e-5) after each class, bond dimension up to 32,
    <Z_i> of every qubit after each step. A step is one Trotter step; the
    unit is Trotter steps/s. Ranks run replicas."""
    import torch

    from dequantizer_b200.workloads import run_eagle_simulation

    n_steps = args.eagle_steps
    torch.cuda.synchronize()
    barrier(world)
    with ClockSampler(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        z, em = run_eagle_simulation(max_chi=32, layers_per_regauging=1, trotter_steps=n_steps, accuracy=1e-5,
                                     theta=0.6, is_infinite=False, colour_classes=True, all_qubits=True,
                                     on_step=profile_hook(args.profile_steps))
        e1.record()
        e1.synchronize()
    elapsed = reduce_max(e0.elapsed_time(e1) * 1e-3, world)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "workload": "kicked Ising, 127-qubit heavy-hex", "value": world * n_steps / elapsed,
            "unit": "Trotter steps/s", "n_gpus": world, "steps": n_steps, "warmup": 0,
            "ms_per_step": elapsed / n_steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"lattice": "heavy-hex, 127 qubits, 144 edges", "chi": 32, "theta": 0.6,
                       "gates": "RX(0.6) on all qubits, RZZ(-pi/2) on all edges in 3 colour classes",
                       "regauge": "after each colour class, BP accuracy 1e-5"},
            "max_bond": int(em._layout.edge_chi.max()),
            "z_mean_final": float(np.mean(z[-1])), "z_target_final": float(z[-1][62]),
            "clocks": clk.summary(),
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["bp", "anneal", "grad", "ising3d", "eagle"], default="bp",
                    help="bp: BP sweep on the 1024-node chi=16 graph (default); anneal: batched annealing; "
                         "grad: gradient of the final annealing energy w.r.t. the schedule; ising3d: 3-D Ising "
                         "canonicalisation; eagle: kicked Ising on the 127-qubit heavy-hex lattice")
    ap.add_argument("--grad-nodes", type=int, default=512)
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--chi", type=int, default=8)
    ap.add_argument("--anneal-precision", choices=["fp64", "mixed"], default="fp64",
                    help="batched annealing: plain FP64, or BF16 tensor-core regauge sweeps handing over to FP64")
    ap.add_argument("--trotter-steps", type=int, default=200)
    ap.add_argument("--eagle-steps", type=int, default=20, help="Trotter steps of the eagle workload")
    ap.add_argument("--profile-steps", default=None,
                    help="A:B -- CUDA profiler range over the timed steps A..B-1 of the anneal and eagle "
                         "workloads (for ncu --profile-from-start off)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=4.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-suite", action="store_true", help="skip the bounded runs of the other workloads")
    ap.add_argument("--anneal-sample", choices=["schedule", "mid"], default="schedule",
                    help="anneal workload: steps along the schedule (default), or the suite's mid-schedule sample "
                         "(warm-up steps of --suite-anneal-warm-dt at s = 0.5, then steps of dt at s = 0.5)")
    ap.add_argument("--suite-anneal-warmup", type=int, default=6)
    ap.add_argument("--suite-anneal-steps", type=int, default=4)
    ap.add_argument("--suite-anneal-warm-dt", type=float, default=1.0)
    ap.add_argument("--suite-eagle-steps", type=int, default=6)
    ap.add_argument("--suite-grad-steps", type=int, default=20,
                    help="Trotter steps of the suite's gradient sample (0 skips it)")
    ap.add_argument("--e2e-chunks", type=int, default=8,
                    help="node ranges the end-to-end sweep streams its host inputs in (1: no overlap)")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--only", choices=["fp64", "fp32", "bf16"], default=None,
                    help="time one precision only (profiling runs); prints a short line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        if args.workload == "anneal":
            run_anneal(args, world, rank, local)
        elif args.workload == "grad":
            run_grad(args, world, rank, local)
        elif args.workload == "ising3d":
            run_ising3d(args, world, rank, local)
        elif args.workload == "eagle":
            run_eagle(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
