"""Host logic of the batched and served modes (CPU): job mixes, wave planning under an HBM
budget, the FIFO replay, and the request loop driven by a stand-in engine."""
import numpy as np

from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import batch, serve


def test_batched_specs_follow_the_mix():
    s1 = batch.batched_specs(64, seed=3)
    s2 = batch.batched_specs(64, seed=3)
    assert [(a.n, a.ppc, a.Te, a.density) for a in s1] == [(b.n, b.ppc, b.Te, b.density) for b in s2]
    assert {s.n for s in s1} <= {65, 129, 257, 513}
    assert all(50 <= s.ppc <= 400 and 1 <= s.Te <= 5 and 1e20 <= s.density <= 1e22 and s.steps == 300 for s in s1)
    assert abs(s1[0].L - (s1[0].n - 1) * 0.01 / 128) < 1e-15


def test_waves_respect_the_budget():
    specs = batch.batched_specs(40, seed=1, ppc_scale=0.2)
    sizes = [batch.bytes_needed(batch.job_config(s)) for s in specs]
    budget = 3 * max(sizes)
    waves = batch.plan_waves(specs, budget)
    assert sorted(k for w in waves for k in w) == list(range(len(specs)))
    for w in waves:
        assert sum(sizes[k] for k in w) <= budget
    # every wave but the last could not take the next job
    assert len(waves) >= sum(sizes) / budget


def test_request_stream():
    reqs = serve.served_requests(300, seed=2)
    t = [r.arrival for r in reqs]
    assert t == sorted(t) and t[0] == 0.0
    assert {r.spec.n for r in reqs} <= {129, 257, 513, 1025}
    assert all(20 <= r.spec.ppc <= 200 and 200 <= r.spec.steps <= 2000 for r in reqs)
    d = np.log10([r.spec.density for r in reqs])
    assert d.min() >= 20 and d.max() <= 22
    # offered load is about 1.5x the assumed capacity
    work = sum(r.spec.particle_steps for r in reqs)
    assert 0.8 < work / t[-1] / (1.5 * serve.B200_CAPACITY) < 1.25


def test_fifo_replay():
    specs = batch.batched_specs(3, seed=0)
    reqs = [serve.Request(a, s, k) for k, (a, s) in enumerate(zip([0.0, 1.0, 10.0], specs))]
    out = serve.fifo_replay(reqs, [5.0, 2.0, 1.0])
    # completions 5, 7, 11 -> latencies 5, 6, 1
    assert abs(out["makespan"] - 11.0) < 1e-12
    assert abs(out["p50"] - 5.0) < 1e-12 and abs(out["mean"] - 4.0) < 1e-12


class FakeJob:
    def __init__(self, eng, spec):
        self.eng, self.spec, self.steps = eng, spec, 0

    def diagnostics(self):
        return {"step": self.steps}

    def destroy(self):
        self.eng.jobs.remove(self)


class FakeEngine:
    def __init__(self):
        self.jobs = []
        self.calls = []
        self.reserved = 0

    def reserve(self, nbytes):
        self.reserved = nbytes

    def step_graph(self, k):
        self.calls.append((k, [j.steps for j in self.jobs]))
        for j in self.jobs:
            j.steps += k

    step = step_graph

    def sync(self):
        pass


class FakeServer(serve.Server):
    def _admit(self, req, now):
        j = FakeJob(self.engine, req.spec)
        self.engine.jobs.append(j)
        return j


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.001
        return self.t

    def sleep(self, dt):
        self.t += dt


def test_server_loop_with_stand_in_engine():
    specs = batch.batched_specs(12, seed=7, ppc_scale=0.05)
    for k, s in enumerate(specs):
        s.steps = 7 + 5 * k
    reqs = [serve.Request(0.002 * k, s, k) for k, s in enumerate(specs)]
    sizes = [batch.bytes_needed(batch.job_config(s)) for s in specs]
    budget = 4 * max(sizes)
    clk = Clock()
    eng = FakeEngine()
    srv = FakeServer(engine=eng, budget_bytes=budget, quantum=6, clock=clk, sleep=clk.sleep)
    out = srv.run(reqs)
    assert eng.reserved == budget   # the budget is mapped into the job pool before the first request
    comp = out["completions"]
    assert [c.index for c in comp] == list(range(len(specs)))
    # every job ran exactly its own number of steps
    assert all(c.diagnostics["step"] == specs[c.index].steps for c in comp)
    # admissions in arrival order, never above the budget
    admits = [e for e in srv.log if e[0] == "admit"]
    assert [e[1] for e in admits] == sorted(e[1] for e in admits)
    assert all(e[4] <= budget for e in srv.log)
    # overlap: at some point several jobs were stepped together
    assert max(len(c[1]) for c in eng.calls) > 1
    assert all(c.finished >= c.admitted >= c.arrival for c in comp)
    assert out["p99"] >= out["p50"] > 0


class _OptEngine:
    """Stand-in engine that keeps the options the tuner sets."""
    def __init__(self):
        self.opts = {}

    def set_option(self, k, v):
        self.opts[k] = v


class _SortJob:
    def __init__(self):
        self.sort_every = None

    def set_sort_every(self, v):
        self.sort_every = v


def test_autotuner_coordinate_search_on_host():
    """The tuner times each knob's candidates with the others at their best so far, keeps the
    fastest, leaves it applied, and stays within half of the steps it may use."""
    from pic_cuda_b200 import autotune
    eng, jobs = _OptEngine(), [_SortJob(), _SortJob()]
    cost = {("lk", 1): 0.5, ("mc", 3): 0.25, ("wt", 4): 0.125}

    class T(autotune.Tuner):
        def _time(self, engine, stream, steps):
            o = engine.opts
            c = 10.0 - cost.get(("lk", o[L.OPT_MG_LEVELS_KERNEL]), 0.0)
            c -= cost.get(("mc", o[L.OPT_MOVER_CTAS_PER_SM]), 0.0)
            c -= cost.get(("wt", o[L.OPT_MG_WIDE_TILES]), 0.0)
            c -= 0.0625 if jobs[0].sort_every == 20 else 0.0
            return c

    t = T(steps_per_trial=3)
    used = t.tune(eng, jobs, None, max_steps=300)
    assert t.chosen == {"levels_kernel": 1, "sort_every": 20, "mover_ctas_per_sm": 3, "mg_wide_tiles": 4}
    assert eng.opts == {L.OPT_MG_LEVELS_KERNEL: 1, L.OPT_MOVER_CTAS_PER_SM: 3, L.OPT_MG_WIDE_TILES: 4}
    assert all(j.sort_every == 20 for j in jobs)
    # one trial for the start point and one per further candidate: 1 + 1 + 1 + 1 + 2
    assert len(t.trials) == 6 and used == 6 * 4
    # a small step budget cuts the search short and stays within half of it
    t2 = T(steps_per_trial=3)
    used2 = t2.tune(_OptEngine(), [_SortJob()], None, max_steps=20)
    assert used2 <= 10 and len(t2.trials) == used2 // 4
