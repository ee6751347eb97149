"""Monte Carlo collisions on the GPU against the oracle (same Philox streams) and against
the expected count n sigma(v) v dt (3 sigma)."""
import math

import numpy as np
import pytest

from pic_cuda_b200 import _lib as L
from pic_cuda_b200 import configs as cf

pytestmark = pytest.mark.gpu


def _by_pid(d):
    o = np.argsort(d["pid"])
    return {k: v[o] for k, v in d.items()}


def test_null_collision_matches_oracle_per_particle(engine, orc):
    n = 200_000
    cfg = cf.plasma(65, 0.01, n, dt=1e-11, mcc=cf.argon_mcc(3.2e21), walls=L.WALLS_NONE)
    cfg.species[0].capacity = cfg.species[1].capacity = n + 50_000
    job = engine.add_job(cfg)
    try:
        cf.load_plasma(job, n, 0.01, 20.0, 0.03, seed=99)  # hot electrons: every process fires
        init = [job.export_species(s) for s in (0, 1)]
        sim = orc.Sim(cfg)
        for s in (0, 1):
            d = init[s]
            sim.load(s, d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["pid"])
        job.run_phases(L.PHASE_MCC, step=0)
        sim.mcc()
        st = sim.stats()
        dg = job.diagnostics()
        for s in (0, 1):
            a, b = _by_pid(job.export_species(s)), _by_pid(sim.export(s))
            assert abs(len(a["pid"]) - len(b["pid"])) <= 2
            common = np.intersect1d(a["pid"], b["pid"])
            ia, ib = np.searchsorted(a["pid"], common), np.searchsorted(b["pid"], common)
            va = np.stack([a["vx"][ia], a["vy"][ia], a["vz"][ia]])
            vb = np.stack([b["vx"][ib], b["vy"][ib], b["vz"][ib]])
            bad = np.linalg.norm(va - vb, axis=0) > 1e-4 * np.linalg.norm(vb, axis=0) + 1e-3
            assert bad.sum() <= max(3, 1e-4 * len(common)), (s, bad.sum())
            for p in range(4):
                assert abs(dg["collisions"][s][p] - st["collisions"][s][p]) <= 3
        assert st["ionizations"] > 100
        assert abs(dg["ionizations"] - st["ionizations"]) <= 2
    finally:
        job.destroy()


def test_collision_count_within_3_sigma(engine):
    n = 1_000_000
    E = np.logspace(-2, 3, 512)
    dens, sig, dt = 3.2e21, 1e-19, 1e-11
    mcc = {"mode": L.MCC_NULL_COLLISION, "density": dens,
           "processes": [(L.PROC_ELASTIC, 0, 0.0, E, np.full(512, sig))], "e_species": 0, "i_species": 1}
    cfg = cf.make_config(65, 0.01, dt, [(-cf.QE, cf.ME, 1.0, n + 1024), (cf.QE, cf.M_AR, 1.0, 1024)], mcc=mcc,
                         walls=L.WALLS_NONE)
    job = engine.add_job(cfg)
    try:
        x, y, vx, vy, vz = cf.maxwellian_state(n, 0.01, 3.0, cf.ME, 21)
        job.load_species(0, x, y, vx, vy, vz)
        v = job.export_species(0)
        speed = np.sqrt(v["vx"] ** 2 + v["vy"] ** 2 + v["vz"] ** 2)
        p = dens * sig * speed * dt  # n sigma(v) v dt
        mu, sd = p.sum(), math.sqrt((p * (1 - p)).sum())
        job.run_phases(L.PHASE_MCC, step=3)
        got = job.diagnostics()["collisions"][0][0]
        assert abs(got - mu) < 3 * sd, (got, mu, sd)
        # elastic: isotropic directions, energy lost only to recoil (2 m / M per collision at most)
        a = job.export_species(0)
        sp2 = np.sqrt(a["vx"] ** 2 + a["vy"] ** 2 + a["vz"] ** 2)
        assert np.all(sp2 <= speed * (1 + 1e-6))
        assert np.all(sp2 >= speed * (1 - 4 * cf.ME / cf.M_AR) - 1e-3)
    finally:
        job.destroy()


def test_reference_elastic_form_statistics(engine):
    # elasticCollisions (mcc.cu:114-150): P = 1 - exp(-n sigma |v| dt), |v| (2D) kept
    n = 400_000
    E = np.logspace(-2, 3, 128)
    dens, sig, dt = 1e21, 2e-19, 1e-10
    mcc = {"mode": L.MCC_REF_ELASTIC2D, "density": dens, "processes": [(L.PROC_ELASTIC, 0, 0.0, E, np.full(128, sig))]}
    cfg = cf.make_config(33, 0.01, dt, [(-cf.QE, cf.ME, 1.0, n + 1024)], mcc=mcc, walls=L.WALLS_NONE)
    job = engine.add_job(cfg)
    try:
        x, y, vx, vy, vz = cf.maxwellian_state(n, 0.01, 3.0, cf.ME, 4)
        job.load_species(0, x, y, vx, vy, vz)
        b = job.export_species(0)
        s2 = np.hypot(b["vx"], b["vy"])
        p = 1 - np.exp(-dens * sig * s2 * dt)
        job.run_phases(L.PHASE_MCC, step=0)
        a = job.export_species(0)
        got = job.diagnostics()["collisions"][0][0]
        assert abs(got - p.sum()) < 3 * math.sqrt((p * (1 - p)).sum())
        np.testing.assert_allclose(np.hypot(a["vx"], a["vy"]), s2, rtol=2e-6)
        np.testing.assert_array_equal(a["vz"], b["vz"])
    finally:
        job.destroy()


def test_file_cross_sections_match_oracle_per_particle(engine, orc):
    """The reference's argon tables (csf/Ar.txt elastic and csf/Ar+.txt ionisation, non-uniform
    energy grids from 0 eV and from 15.76 eV, committed as tests/golden/csf_argon.npz) in the
    null-collision engine: the table lookup takes its bisection branch.  Per particle against
    the oracle on the same Philox streams, as the synthetic-table test above."""
    from pathlib import Path
    from pic_cuda_b200 import xs
    g = np.load(Path(__file__).resolve().parent / "golden" / "csf_argon.npz")
    mcc = xs.argon_file_mcc(3.2e21, (g["elastic_E"], g["elastic_sigma"]), (g["ionization_E"], g["ionization_sigma"]))
    n = 200_000
    cfg = cf.plasma(65, 0.01, n, dt=1e-11, mcc=mcc, walls=L.WALLS_NONE)
    cfg.species[0].capacity = cfg.species[1].capacity = n + 50_000
    job = engine.add_job(cfg)
    try:
        cf.load_plasma(job, n, 0.01, 25.0, 0.03, seed=17)  # hot electrons: ionisation fires
        init = [job.export_species(s) for s in (0, 1)]
        sim = orc.Sim(cfg)
        for s in (0, 1):
            d = init[s]
            sim.load(s, d["x"], d["y"], d["vx"], d["vy"], d["vz"], d["pid"])
        sim.set_counters(5, job.diagnostics()["next_pid"])
        job.run_phases(L.PHASE_MCC, step=5)
        sim.mcc()
        st = sim.stats()
        dg = job.diagnostics()
        for s in (0, 1):
            a, b = _by_pid(job.export_species(s)), _by_pid(sim.export(s))
            assert abs(len(a["pid"]) - len(b["pid"])) <= 2
            common = np.intersect1d(a["pid"], b["pid"])
            ia, ib = np.searchsorted(a["pid"], common), np.searchsorted(b["pid"], common)
            va = np.stack([a["vx"][ia], a["vy"][ia], a["vz"][ia]])
            vb = np.stack([b["vx"][ib], b["vy"][ib], b["vz"][ib]])
            bad = np.linalg.norm(va - vb, axis=0) > 3e-4 * np.linalg.norm(vb, axis=0) + 1e-3
            assert bad.sum() <= max(3, 1e-4 * len(common)), (s, bad.sum())
            for p in range(4):
                assert abs(dg["collisions"][s][p] - st["collisions"][s][p]) <= 3, (s, p)
        assert st["collisions"][0][0] > 1000          # elastic from Ar.txt
        assert st["ionizations"] > 100                 # ionisation from Ar+.txt
        assert abs(dg["ionizations"] - st["ionizations"]) <= 2
    finally:
        job.destroy()
