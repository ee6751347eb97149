"""Headless snapshot of particle positions (the reference's vertex-buffer fill,
convertPositionsToFloat, kernels.cu:268-274) and of the diagnostics, against the FP64 export
of the same state: every FP32 value is the FP64 position rounded once."""
import numpy as np
import pytest

from pic_cuda_b200 import configs as cf

pytestmark = pytest.mark.gpu


def test_snapshot_positions_equal_rounded_export(engine, tmp_path):
    n = 50_000
    cfg = cf.plasma(129, 0.01, n, tol=1e-6, mcc=cf.argon_mcc(3.2e21))
    job = engine.add_job(cfg)
    try:
        cf.load_plasma(job, n, 0.01, 2.0, 0.03, seed=17)
        engine.step(3)
        for s in (0, 1):
            e = job.export_species(s)
            ref = np.stack([e["x"], e["y"]], axis=1).astype(np.float32)
            host = job.snapshot_positions(s)
            dev = job.snapshot_positions(s, device=True).cpu().numpy()
            assert host.shape == ref.shape == dev.shape and len(ref) > 0.9 * n
            assert np.array_equal(host, ref) and np.array_equal(dev, ref)
        path = tmp_path / "frame.npz"
        job.write_snapshot(path)
        f = np.load(path)
        assert np.array_equal(f["xy0"], job.snapshot_positions(0))
        assert int(f["diag_step"]) == 3
    finally:
        job.destroy()
