"""Autotuner for a batch of jobs: picks the engine's multigrid launch shape
(PIC_OPT_MG_LEVELS_KERNEL: one launch per level, or levels 1..lc as one cooperative launch)
and the counting-sort cadence of the jobs by timing a few real steps of each candidate.

Tuning steps are ordinary steps of the jobs (results do not depend on the launch shape; with
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

    def tune(self, engine, jobs, stream, max_steps: int) -> int:
        """Runs the trials on the jobs and leaves the fastest settings in place; returns the
        number of steps the trials took."""
        per = self.steps_per_trial + 1
        cands = [(lk, se) for lk in self.levels_kernel for se in self.sort_every]
        if len(cands) * per > max_steps // 2:
            cands = cands[: max(1, (max_steps // 2) // per)]
        best = None
        for lk, se in cands:
            engine.set_option(L.OPT_MG_LEVELS_KERNEL, lk)
            for j in jobs:
                j.set_sort_every(se)
            ms = self._time(engine, stream, self.steps_per_trial)
            self.trials.append({"levels_kernel": lk, "sort_every": se, "ms_per_step": ms})
            if best is None or ms < best[0]:
                best = (ms, lk, se)
        _, lk, se = best
        engine.set_option(L.OPT_MG_LEVELS_KERNEL, lk)
        for j in jobs:
            j.set_sort_every(se)
        self.chosen = {"levels_kernel": lk, "sort_every": se}
        return len(cands) * per
