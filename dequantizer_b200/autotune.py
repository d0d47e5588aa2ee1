"""Autotuner for the launch shapes of the gauge and gate kernels.

Knobs (``dqz_set_tuning``, include/dqz.h): warps per CTA of the one-warp
``vidal_edges`` / ``vidal_distance`` kernels, the one-warp vs one-CTA gauge
path, and the grid of ``simple_update``. A knob changes scheduling only, never
the per-item arithmetic, so results are bit-identical for every setting.

``Tuner.tune`` times each candidate with CUDA events on the caller's own
arenas (median of ``reps`` runs after one warm-up), keeps the fastest, writes
it to a JSON cache keyed by device name, kernel family and shape, and applies
it. Later calls with the same key read the cache and time nothing. The cache
file is ``$DQZ_TUNE_CACHE`` or ``~/.cache/dequantizer_b200/tuning.json``.
"""

import json
import os
from typing import Callable, Dict, List, Optional

import torch

from . import _lib

KNOBS = {"gauge_edge_warps": 0, "gauge_dist_warps": 1, "gauge_path": 2, "su_grid": 3, "su_onchip": 4,
         "sweep_onecta": 5}


def set_knobs(cfg: Dict[str, int]) -> None:
    for name, value in cfg.items():
        _lib.call("dqz_set_tuning", KNOBS[name], int(value))


def get_knobs() -> Dict[str, int]:
    return {name: int(_lib.lib().dqz_get_tuning(k)) for name, k in KNOBS.items()}


def default_cache_path() -> str:
    return os.environ.get("DQZ_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "dequantizer_b200", "tuning.json"))


class Tuner:
    def __init__(self, path: Optional[str] = None, reps: int = 5, timer: Optional[Callable] = None):
        self.path = path or default_cache_path()
        self.reps = int(reps)
        self.timer = timer or self._cuda_time
        self.cache: Dict[str, Dict[str, int]] = {}
        if os.path.exists(self.path):
            with open(self.path) as f:
                self.cache = json.load(f)
        self.timed_keys: List[str] = []

    @staticmethod
    def key(kind: str, device_name: str, **shape) -> str:
        return "|".join([device_name, kind] + ["%s=%s" % (k, shape[k]) for k in sorted(shape)])

    def _cuda_time(self, run: Callable[[], None]) -> float:
        run()  # warm-up (also lets one-time kernel attributes settle)
        times = []
        for _ in range(self.reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        times.sort()
        return times[len(times) // 2]

    def tune(self, key: str, candidates: List[Dict[str, int]], run: Callable[[], None]) -> Dict[str, int]:
        """Best of ``candidates`` for ``run`` (cached by ``key``), applied."""
        if key in self.cache:
            set_knobs(self.cache[key])
            return self.cache[key]
        before = get_knobs()
        best, best_t = None, float("inf")
        for cfg in candidates:
            set_knobs({**before, **cfg})
            t = self.timer(run)
            if t < best_t:
                best, best_t = cfg, t
        self.cache[key] = dict(best)
        self.timed_keys.append(key)
        self._save()
        set_knobs({**before, **best})
        return best

    def _save(self) -> None:
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.cache, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def _device_name(device) -> str:
    return torch.cuda.get_device_name(device) if torch.cuda.is_available() else "cpu"


def tune_gauge(layout, T, n2e, eps: float = 1e-10, tuner: Optional[Tuner] = None) -> Dict[str, int]:
    """Vidal-gauge + Vidal-distance launch shapes for this layout's shapes
    (max bond, max degree, max bond slice, node count bucket)."""
    from .maps import vidal_distance_partial, vidal_gauge_packed

    tuner = tuner or Tuner()
    chi, slc = layout.max_chi(), layout.max_slice()
    deg = int(layout.degree.max(initial=0))
    bucket = 1 << max(0, int(layout.n_nodes).bit_length() - 1)
    key = tuner.key("gauge", _device_name(layout.device), chi=chi, deg=deg, slice=slc, nodes=bucket)
    G0, lam0 = vidal_gauge_packed(layout, T, n2e, eps)
    orth = torch.empty(max(layout.msg_elems, 1), dtype=torch.complex128, device=layout.device)
    part = torch.empty(max(layout.n_halves, 1), dtype=torch.float64, device=layout.device)

    def run():
        vidal_gauge_packed(layout, T, n2e, eps, out=(G0, lam0, orth))
        vidal_distance_partial(layout, G0, lam0, eps, part)

    candidates = [{"gauge_path": 2, "gauge_edge_warps": 0, "gauge_dist_warps": 0}]
    if chi <= 16:
        for we in (1, 2, 4, 8):
            for wd in (1, 2, 4, 8):
                candidates.append({"gauge_path": 1, "gauge_edge_warps": we, "gauge_dist_warps": wd})
    return tuner.tune(key, candidates, run)
