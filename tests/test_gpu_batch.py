"""Jobs stepped together in one engine give the same result as each job alone.
With the int64 deposit the whole step is order independent, so the check is bit-exact."""
import numpy as np
import pytest

from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf
from pic_cuda_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _by_pid(d):
    o = np.argsort(d["pid"])
    return {k: v[o] for k, v in d.items()}


def _jobs():
    a = cf.plasma(65, 0.005, 20_000, deposit=L.DEPOSIT_I64, sort_every=2, seed=11, tol=1e-9,
                  mcc=cf.argon_mcc(3.2e21))
    b = cf.plasma(129, 0.01, 30_000, deposit=L.DEPOSIT_I64, sort_every=3, seed=12, tol=1e-9)
    c = cf.plasma(257, 0.02, 40_000, deposit=L.DEPOSIT_I64, sort_every=5, seed=13, tol=1e-9,
                  mcc=cf.argon_mcc(1e21))
    return [(a, 0.005, 5.0, 100), (b, 0.01, 2.0, 101), (c, 0.02, 3.0, 102)]


def _run(engine, specs, steps):
    jobs = []
    for cfg, Ld, Te, seed in specs:
        j = engine.add_job(cfg)
        n = cfg.species[0].capacity * 4 // 5 - 1024
        cf.load_plasma(j, int(n), Ld, Te, 0.03, seed=seed)
        jobs.append(j)
    engine.step(steps)
    return [([_by_pid(j.export_species(s)) for s in (0, 1)], j.get_grid(L.GRID_PHI), j.diagnostics()) for j in jobs]


def test_batch_equals_alone_bitwise():
    specs = _jobs()
    e = Engine(0)
    together = _run(e, specs, 6)
    e.close()
    for k, spec in enumerate(specs):
        e = Engine(0)
        alone = _run(e, [spec], 6)[0]
        e.close()
        t = together[k]
        for s in (0, 1):
            for key in ("pid", "x", "y", "vx", "vy", "vz"):
                assert np.array_equal(t[0][s][key], alone[0][s][key]), (k, s, key)
        assert np.array_equal(t[1], alone[1])
        assert t[2]["vcycles"] == alone[2]["vcycles"]
    assert together[0][2]["step"] == 6


def test_repeat_run_bitwise_identical():
    specs = _jobs()[:1]
    e = Engine(0)
    r1 = _run(e, specs, 4)
    e.close()
    e = Engine(0)
    r2 = _run(e, specs, 4)
    e.close()
    for s in (0, 1):
        for key in ("pid", "x", "y", "vx", "vy", "vz"):
            assert np.array_equal(r1[0][0][s][key], r2[0][0][s][key])


def test_graph_step_equals_stream_step_bitwise():
    """pic_step_graph (CUDA graph, V-cycle loop as a conditional WHILE node) gives exactly
    the state pic_step (host-driven loop) gives."""
    specs = _jobs()
    res = []
    for use_graph in (False, True):
        e = Engine(0)
        jobs = []
        for cfg, Ld, Te, seed in specs:
            j = e.add_job(cfg)
            n = cfg.species[0].capacity * 4 // 5 - 1024
            cf.load_plasma(j, int(n), Ld, Te, 0.03, seed=seed)
            jobs.append(j)
        for _ in range(7):  # crosses sort steps of every job
            (e.step_graph if use_graph else e.step)(1)
        res.append([([_by_pid(j.export_species(s)) for s in (0, 1)], j.get_grid(L.GRID_PHI), j.diagnostics())
                    for j in jobs])
        e.close()
    for a, b in zip(res[0], res[1]):
        for s in (0, 1):
            for key in ("pid", "x", "y", "vx", "vy", "vz"):
                assert np.array_equal(a[0][s][key], b[0][s][key]), (s, key)
        assert np.array_equal(a[1], b[1])
        assert a[2]["vcycles"] == b[2]["vcycles"] and a[2]["step"] == b[2]["step"] == 7


def test_multi_wave_grid_repeatable_bitwise():
    """At 1025^2 the level-0 multigrid kernels run in more than one wave of CTAs, so a tile
    that starts late sees neighbours that already finished.  Two runs (stream-ordered and
    graph) of the same job must agree bit for bit, which they do only if no kernel reads a
    halo that another CTA of the same launch overwrites."""
    cfg = cf.plasma(1025, 0.05, 200_000, deposit=L.DEPOSIT_I64, seed=31, tol=1e-9, warm_start=1)
    out = []
    for use_graph in (False, True, True):
        e = Engine(0)
        j = e.add_job(cfg)
        cf.load_plasma(j, 200_000, 0.05, 3.0, 0.03, seed=32)
        for _ in range(3):
            (e.step_graph if use_graph else e.step)(1)
        out.append((j.get_grid(L.GRID_PHI), j.diagnostics()["vcycles"]))
        e.close()
    for phi, cyc in out[1:]:
        assert np.array_equal(phi, out[0][0]) and cyc == out[0][1]


@pytest.mark.parametrize("opts", [
    {L.OPT_MOVER_CTAS_PER_SM: 1},
    {L.OPT_MOVER_CTAS_PER_SM: 3, L.OPT_MG_WIDE_TILES: 0},
    {L.OPT_MG_WIDE_TILES: 64, L.OPT_MG_LEVELS_KERNEL: 1},
])
def test_tuning_options_bitwise_identical(opts):
    """The launch shapes the autotuner chooses among (CTAs per SM of the particle pass, CTA
    size of the multigrid tile levels, one launch per level or the cooperative levels kernel)
    change no result: with the int64 deposit every step is bit for bit the default's."""
    specs = _jobs()
    e = Engine(0)
    ref = _run(e, specs, 5)
    e.close()
    e = Engine(0)
    for k, v in opts.items():
        e.set_option(k, v)
        assert e.get_option(k) == v
    got = _run(e, specs, 5)
    e.close()
    for a, b in zip(ref, got):
        for s in (0, 1):
            for key in ("pid", "x", "y", "vx", "vy", "vz"):
                assert np.array_equal(a[0][s][key], b[0][s][key]), (s, key)
        assert np.array_equal(a[1], b[1])
        assert a[2]["vcycles"] == b[2]["vcycles"]


def test_due_sort_leaves_ordered_slots_alone():
    """A counting sort that falls due reorders a slot whose particles are out of cell order and
    leaves one where fewer than 1/32 of them follow a particle of a later cell.  Electrons
    loaded at random positions come out of the step (sorted before the first particle pass and
    at its end) with few descents; ions loaded in cell order with 1% of them swapped far apart
    (2% descents), cold enough not to change cell, keep their exact order through the step,
    swapped pairs included."""
    n, nx, L_dom = 20_000, 129, 0.01
    cfg = cf.plasma(nx, L_dom, n, sort_every=1, seed=3, tol=1e-6)
    ncx = nx - 1
    dx = L_dom / ncx

    def keys(cell):
        c = cell.astype(np.int64) & 0xFFFFFFFF
        return (c >> 16) * ncx + (c & 0xFFFF)

    ex, ey, evx, evy, evz = cf.maxwellian_state(n, L_dom, 5.0, cf.ME, 7)
    ix, iy, ivx, ivy, ivz = cf.maxwellian_state(n, L_dom, 1e-6, cf.M_AR, 8)
    order = np.argsort(np.floor(iy / dx) * ncx + np.floor(ix / dx), kind="stable")
    rng = np.random.default_rng(9)
    a = rng.choice(n // 2, n // 200, replace=False)
    b = a + n // 2
    order[a], order[b] = order[b].copy(), order[a].copy()
    ix, iy, ivx, ivy, ivz = (v[order] for v in (ix, iy, ivx, ivy, ivz))
    ipid = np.arange(n, dtype=np.uint32) + 1_000_000
    e = Engine(0)
    try:
        job = e.add_job(cfg)
        job.load_species(0, ex, ey, evx, evy, evz)
        job.load_species(1, ix, iy, ivx, ivy, ivz, ipid)
        before = keys(job.export_raw(1)["cell"].cpu().numpy())
        desc_before = np.count_nonzero(np.diff(before) < 0)
        assert 0 < desc_before < n // 32
        e.step(1)
        ri = job.export_raw(1)
        assert np.array_equal(ri["pid"].cpu().numpy().astype(np.uint32), ipid)   # not reordered
        assert np.array_equal(keys(ri["cell"].cpu().numpy()), before)           # nor moved
        ke = keys(job.export_raw(0)["cell"].cpu().numpy())
        assert np.count_nonzero(np.diff(ke) < 0) < len(ke) // 10                 # sorted this step
    finally:
        e.close()
