"""Launch-configuration autotuner for the batched solver.

The solver kernels come in two builds with different shapes on the SM: the default build runs
two instances (CTAs of 256 threads, 83 KB of shared memory) per SM and does the FP32 factor's
update tiles on FFMA, and the tensor-core build runs one per SM (a kernel holding tcgen05
instructions is scheduled one CTA per SM) with those tiles on tcgen05.  Which one is faster, and
whether a second resident instance pays for sharing the SM, depends on the fronts: large fronts
are dominated by their update tiles, small ones by latency-bound vector work.  `tune` decides by
timed trial launches on a sample of the workload itself, the same launch the caller makes, and
returns the fastest candidate with every trial's time.

    from mumblebee_b200.autotune import tune
    choice = tune(probs, IPMSettings(precision="mixed"))
    Batch(probs, choice.settings).run(grid=choice.grid)
"""
from __future__ import annotations

import dataclasses
import statistics
from dataclasses import dataclass, field

import numpy as np

from .ipm import Batch, IPMSettings

# (name, settings.fp32_tiles, resident instances per SM); the tensor-core build fits one per SM
CANDIDATES = (("ffma_2_per_sm", 1, 2), ("ffma_1_per_sm", 1, 1), ("tcgen05_1_per_sm", 2, 1))


@dataclass
class Choice:
    name: str
    settings: IPMSettings
    grid: int                       # CTAs of the persistent launch
    trials: dict = field(default_factory=dict)   # candidate -> mean ms per sampled instance
    sample: int = 0
    nsm: int = 0

    def as_dict(self):
        return {"choice": self.name, "fp32_tiles": self.settings.fp32_tiles, "grid": self.grid,
                "sample_instances": self.sample, "ms_per_instance": self.trials}


def largest_front(prob) -> int:
    s = prob.symbolic()
    r = np.asarray(s["nres"]) + np.asarray(s["nsep"])
    return int(r.max()) if r.size else 0


def _sample(probs, size, seed):
    """A sample of `size` instances stratified by largest front (the quantity the candidates
    differ on): instances sorted by it and taken at evenly spaced ranks."""
    if len(probs) <= size:
        return list(probs)
    order = np.argsort([largest_front(p) for p in probs], kind="stable")
    rng = np.random.default_rng(seed)
    pick = np.linspace(0, len(probs) - 1, size).round().astype(int)
    pick = np.unique(np.clip(pick + rng.integers(0, 2, size), 0, len(probs) - 1))
    return [probs[i] for i in order[pick]]


def tune(probs, settings: IPMSettings | None = None, nsm: int = 148, sample: int = 0, repeats: int = 2,
         seed: int = 0, candidates=CANDIDATES) -> Choice:
    """Time each candidate launch configuration on a sample of `probs` (by default eight instances
    per SM: a persistent CTA then runs several instances, as in a large batch, so that the trial
    measures throughput rather than the latency of one instance per CTA) and return the fastest.
    An FP64 factor never runs the FP32 tiles, so for precision "fp64" only the resident-instance
    count is tuned.  Each trial is a warm-up launch and `repeats` timed launches (CUDA events)."""
    settings = settings or IPMSettings()
    sub = _sample(probs, sample or 8 * nsm, seed)
    trials, best = {}, None
    for name, tiles, per_sm in candidates:
        if settings.precision == "fp64" and tiles == 2:
            continue
        st = dataclasses.replace(settings, fp32_tiles=tiles)
        grid = min(len(sub), nsm * per_sm)
        b = Batch(sub, st)
        b.run(grid=grid)
        ms = statistics.mean(b.run(grid=grid) for _ in range(repeats))
        del b
        trials[name] = ms / len(sub)
        if best is None or trials[name] < trials[best[0]]:
            best = (name, st, per_sm)
    name, st, per_sm = best
    return Choice(name, st, min(len(probs), nsm * per_sm), trials, len(sub), nsm)
