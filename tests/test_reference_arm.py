"""Host logic of bench.py's CPU arm (`--impl reference` and the bench line's
cpu_baseline): whole steps of the two-species bounded plasma through the
oracle, on a small sub-domain here (CPU only)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_cpu_arm_runs_whole_steps_with_the_gpu_stopping_rule():
    run = bench.CpuRun(16, 8, seed=3)
    assert run.n_total == 2 * 16 * 16 * 8
    for _ in range(3):
        run.step()
    # the solve of every step stops by the GPU backends' rule: relative residual 1e-8 within 16 cycles
    assert run.last["rel_residual"] <= 1e-8
    assert 1 <= run.last["batches"] <= 8
    # grounded walls: phi vanishes on the fixed nodes (to the solve's tolerance)
    assert np.abs(run.phi[run.fixed]).max() <= 1e-8 * np.abs(run.phi).max()
    for q, m, pos, vel in run.species:
        alive = ~np.isnan(pos[0])
        assert alive.sum() > 0.9 * pos.shape[1]                           # few particles reach a wall
        assert np.all((pos[:, alive] >= 0.0) & (pos[:, alive] < 16.0))   # absorbed ones are marked NaN
        assert np.all(np.isfinite(vel[:, alive]))
    text = run.describe(3)
    assert "3 whole steps" in text and "16x16-cell" in text


def test_cpu_baseline_line_fields():
    # the reported baseline is measured whole steps (no extrapolation): value = particles x steps / seconds
    bench_cells = bench.CPU_CELLS
    try:
        bench.CPU_CELLS = 16
        line = bench.cpu_baseline(8, warmup=1, steps=2)
    finally:
        bench.CPU_CELLS = bench_cells
    assert line["kind"] == "port" and line["unit"] == "particle-steps/s"
    assert line["value"] > 0 and line["cores"] >= 1
    assert "2 whole steps" in line["sample"]
