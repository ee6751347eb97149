"""Served and batched modes on the GPU: a request's result is the same alone and in the mix
(bit for bit with the int64 deposit), and batched waves run every job to its step count."""
import numpy as np
import pytest

from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import autotune, batch, serve

pytestmark = pytest.mark.gpu


def _by_pid(d):
    o = np.argsort(d["pid"])
    return {k: v[o] for k, v in d.items()}


def test_served_results_equal_alone():
    import torch
    from pic_cuda_b200.engine import Engine
    specs = [batch.JobSpec(n=n, ppc=2, Te=te, density=dens, steps=st, seed=900 + k, deposit=L.DEPOSIT_I64)
             for k, (n, te, dens, st) in enumerate([(129, 2.0, 3e21, 23), (257, 4.0, 1e21, 31),
                                                     (129, 1.5, 8e21, 17), (257, 3.0, 5e20, 12)])]
    reqs = [serve.Request(0.001 * k, s, k) for k, s in enumerate(specs)]
    eng = Engine(0)
    srv = serve.Server(engine=eng, budget_bytes=64 << 30, quantum=5, device=torch.device("cuda", 0),
                       keep_results=True)
    out = srv.run(reqs)
    eng.close()
    assert max(e[3] for e in srv.log if e[0] == "admit") > 1  # requests overlapped on the device
    for c in out["completions"]:
        _, diag, alone = serve.run_alone(specs[c.index], keep_result=True)
        assert c.diagnostics["step"] == diag["step"] == specs[c.index].steps
        assert np.array_equal(c.result["phi"], alone["phi"])
        for s in (0, 1):
            a, b = _by_pid(c.result["species"][s]), _by_pid(alone["species"][s])
            for key in ("pid", "x", "y", "vx", "vy", "vz"):
                assert np.array_equal(a[key], b[key]), (c.index, s, key)


def test_batched_waves_run_every_job():
    specs = batch.batched_specs(6, seed=11, ppc_scale=0.01, steps=40)
    sizes = [batch.bytes_needed(batch.job_config(s)) for s in specs]
    budget = max(sizes)  # the largest job fills a wave by itself
    tuner = autotune.Tuner(steps_per_trial=3)
    res = batch.run_batched(specs, budget, tuner=tuner)
    assert res.waves >= 2 and len(res.per_job) == len(specs)
    assert sorted(k for k, _ in res.per_job) == list(range(len(specs)))
    assert all(d["step"] == 40 for _, d in res.per_job)
    assert tuner.chosen and len(tuner.trials) >= 2
    assert res.seconds > 0 and res.rate > 0


def test_engine_reserve_maps_pool_memory():
    """pic_engine_reserve maps memory into the job pool once: the device's free memory drops
    by at least the reservation, job creation afterwards takes no more from the device, and a
    negative size is rejected."""
    import torch
    from pic_cuda_b200.engine import Engine
    eng = Engine(0)
    try:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        eng.reserve(2 << 30)
        free1, _ = torch.cuda.mem_get_info(0)
        assert free0 - free1 >= 2 << 30
        spec = batch.JobSpec(n=257, ppc=4, Te=2.0, density=1e21, steps=2, seed=5)
        assert batch.bytes_needed(batch.job_config(spec)) < 1 << 30
        job = eng.add_job(batch.job_config(spec))
        torch.cuda.synchronize()
        free2, _ = torch.cuda.mem_get_info(0)
        assert free2 >= free1 - (64 << 20)   # the job's arrays came from the reserved pool
        job.destroy()
        with pytest.raises(L.PicError):
            eng.reserve(-1)
    finally:
        eng.close()
