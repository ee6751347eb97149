"""Autotuner for a batch of jobs: picks, by timing a few real steps of each candidate,
  * the multigrid launch shape (PIC_OPT_MG_LEVELS_KERNEL: one launch per level, or levels
    1..lc as one cooperative launch),
  * the counting-sort cadence of the jobs,
  * the CTAs per SM of the persistent particle pass (PIC_OPT_MOVER_CTAS_PER_SM),
  * which multigrid levels run a tile per 1024-thread CTA (PIC_OPT_MG_WIDE_TILES).
The knobs are tuned in turn (coordinate search): each knob's candidates are timed with the
others at their best so far, and the fastest is kept.

Tuning steps are ordinary steps of the jobs (results do not depend on the launch shapes; with
the int64 deposit they do not depend on the sort cadence either), so they count towards the
jobs' step totals.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import _lib as L


@dataclass
class Tuner:
    levels_kernel: tuple = (0, 1)
    sort_every: tuple = (10, 20)
    mover_ctas_per_sm: tuple = (0, 3)      # 0: as many as fit (4 at 64 registers)
    mg_wide_tiles: tuple = (2, 0, 4)
    steps_per_trial: int = 6
    chosen: dict = field(default_factory=dict)
    trials: list = field(default_factory=list)

    def _time(self, engine, stream, steps: int) -> float:
        import torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        engine.step_graph(1, stream=stream.cuda_stream)  # rebuilds the graph for the new settings
        torch.cuda.synchronize()
        e0.record(stream)
        engine.step_graph(steps, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    @staticmethod
    def _apply(engine, jobs, s: dict) -> None:
        engine.set_option(L.OPT_MG_LEVELS_KERNEL, s["levels_kernel"])
        engine.set_option(L.OPT_MOVER_CTAS_PER_SM, s["mover_ctas_per_sm"])
        engine.set_option(L.OPT_MG_WIDE_TILES, s["mg_wide_tiles"])
        for j in jobs:
            j.set_sort_every(s["sort_every"])

    def tune(self, engine, jobs, stream, max_steps: int) -> int:
        """Runs the trials on the jobs and leaves the fastest settings in place; returns the
        number of steps the trials took (at most half of max_steps)."""
        per = self.steps_per_trial + 1
        budget = max(1, (max_steps // 2) // per)
        knobs = [("levels_kernel", self.levels_kernel), ("sort_every", self.sort_every),
                 ("mover_ctas_per_sm", self.mover_ctas_per_sm), ("mg_wide_tiles", self.mg_wide_tiles)]
        best = {k: v[0] for k, v in knobs}
        timed = {}
        used = 0

        def trial(s):
            key = tuple(sorted(s.items()))
            if key not in timed:
                self._apply(engine, jobs, s)
                timed[key] = self._time(engine, stream, self.steps_per_trial)
                self.trials.append({**s, "ms_per_step": timed[key]})
            return timed[key]

        best_ms = trial(best)
        used += 1
        for name, values in knobs:
            for v in values[1:]:
                if used >= budget:
                    break
                cand = {**best, name: v}
                ms = trial(cand)
                used += 1
                if ms < best_ms:
                    best, best_ms = cand, ms
        self._apply(engine, jobs, best)
        self.chosen = dict(best)
        return used * per
