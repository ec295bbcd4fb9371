"""The run driver on the GPU: a forced, damped fixed-step run advances in
multistep segments yet gives exactly the state of a per-step loop with the
same ring phases; events write the reference's files; a run resumed from
its checkpoint continues the uninterrupted one bit for bit; the adaptive
(CFL) mode reaches t_end."""

import math

import numpy as np
import pytest
import torch
import yaml

pytestmark = pytest.mark.gpu
DT = 2.0**-9  # exact in binary: step times add up without rounding, so no step is clamped

BASE = {
    "grid": {"N": 64, "L": 2 * math.pi},
    "solver": {"alpha": 1.0, "dissipation": {"nu_p": 1e-12, "p": 8},
               "damping": {"type": "linear_drag", "mu": 0.1},
               "time_integration": {"dt": DT, "adaptive_cfl": False}},
    "forcing": {"type": "ring", "kf": 8.0, "dk": 1.0, "epsilon": 0.1, "seed": 7},
    "simulation": {"t_end": 50 * DT, "output_interval": 0.05, "checkpoint_interval": 0.05, "log_interval": 0.02},
    "initial_condition": {"type": "random", "seed": 3},
    "output": {"fields": ["theta", "velocity", "streamfunction"]},
}


@pytest.fixture(scope="module", autouse=True)
def _built():
    from pygsquig_b200.build import build

    build()


def _write(tmp_path, cfg, name="c.yml"):
    p = tmp_path / name
    p.write_text(yaml.safe_dump(cfg))
    return str(p)


def _per_step(cfg_dict, steps):
    from pygsquig_b200 import CombinedDamping, RingForcing, gSQGSolver, make_grid

    g = make_grid(64, 2 * math.pi)
    s = gSQGSolver(g, 1.0, 1e-12, 8)
    st = s.initialize(seed=3)
    ring = RingForcing(kf=8.0, dk=1.0, epsilon=0.1)
    damp = CombinedDamping(mu=0.1, kf=8.0, nu_p=1e-12, p=8)
    rng = np.random.default_rng(7)
    t_end = cfg_dict["simulation"]["t_end"]
    while st["time"] < t_end:  # run.py's loop: dt clamped to the end time
        dt = min(DT, t_end - st["time"])
        st = s.step(st, dt, forcing=ring.bind(rng.uniform(0, 2 * math.pi, ring.n_modes(g)), dt, g), damping=damp)
    assert st["step"] == steps
    return st


def test_segments_equal_per_step_loop_and_files(tmp_path):
    from pygsquig_b200.io import load_checkpoint, load_diagnostics, load_output
    from pygsquig_b200.run import run

    out = tmp_path / "out"
    st = run(_write(tmp_path, BASE), output_dir=str(out))
    ref = _per_step(BASE, st["step"])
    assert st["step"] == 50 and st["time"] == 50 * DT
    assert torch.equal(st["theta_hat"], ref["theta_hat"])
    ck = {p.name for p in (out / "checkpoints").iterdir()}
    assert ck == {"step_00000026.npz", "final_step_00000050.npz"}, ck
    s2, c2 = load_checkpoint(out / "checkpoints" / "final_step_00000050.npz")
    assert torch.equal(s2["theta_hat"], st["theta_hat"].cpu()) and c2.forcing.seed == 7
    d = load_diagnostics(out / "diagnostics" / "timeseries.npz")
    assert len(d["time"]) >= 4 and np.all(np.diff(d["time"]) > 0) and np.all(d["energy"] > 0)
    fields = sorted((out / "fields").iterdir())
    o = load_output(fields[0])
    assert {"theta", "u", "v", "streamfunction"} <= set(o) and o["theta"].shape == (64, 64)
    assert (out / "config.yml").exists() and any((out / "logs").iterdir())


def test_resume_from_checkpoint_continues_run(tmp_path):
    from pygsquig_b200.run import run

    cfg = dict(BASE)
    cfg.pop("forcing")  # phases restart from the seed on resume; without forcing the run is deterministic
    cfg["simulation"] = dict(BASE["simulation"], t_end=30 * DT, checkpoint_interval=0.03)
    full = run(_write(tmp_path, cfg), output_dir=str(tmp_path / "a"))
    half = dict(cfg, simulation=dict(cfg["simulation"], t_end=15 * DT))
    run(_write(tmp_path, half, "h.yml"), output_dir=str(tmp_path / "b"))
    ck = tmp_path / "b" / "checkpoints" / "final_step_00000015.npz"
    resumed = run(_write(tmp_path, cfg, "r.yml"), checkpoint=str(ck), output_dir=str(tmp_path / "c"))
    assert resumed["step"] == full["step"] == 30
    assert torch.equal(resumed["theta_hat"], full["theta_hat"])


def test_adaptive_mode_reaches_t_end(tmp_path):
    from pygsquig_b200.run import run

    cfg = dict(BASE, solver=dict(BASE["solver"], time_integration={"adaptive_cfl": True, "dt_max": 0.01}))
    cfg["simulation"] = dict(BASE["simulation"], t_end=0.05)
    st = run(_write(tmp_path, cfg), output_dir=str(tmp_path / "o"), precision="float32", scheme="ifrk4")
    assert abs(st["time"] - 0.05) < 1e-12 and st["theta_hat"].dtype == torch.complex64
    assert bool(torch.isfinite(torch.view_as_real(st["theta_hat"])).all())


def test_scalar_run_writes_scalar_fields(tmp_path):
    """A run with passive scalars (the reference's scalars section): the
    checkpoint carries the scalar spectra and the field output the scalar
    fields; a zero-diffusivity scalar's mean is conserved."""
    from pygsquig_b200.io import load_checkpoint, load_output
    from pygsquig_b200.run import run

    cfg = dict(BASE, output={"fields": ["theta", "scalars"]})
    cfg["scalars"] = {"enabled": True, "species": [
        {"name": "dye", "kappa": 0.0, "initial_condition": "gaussian", "initial_params": {"width": 0.5}},
        {"name": "salt", "kappa": 1e-3, "initial_condition": "uniform", "initial_params": {"value": 2.0}}]}
    cfg["simulation"] = dict(BASE["simulation"], t_end=20 * DT, output_interval=0.02, checkpoint_interval=0.02)
    out = tmp_path / "s"
    st = run(_write(tmp_path, cfg), output_dir=str(out))
    assert st["step"] == 20 and set(st["scalar_state"].scalars) == {"dye", "salt"}
    ck, _ = load_checkpoint(out / "checkpoints" / "final_step_00000020.npz")
    dye0 = ck["scalar_state"].scalars["dye"]
    x = np.arange(64) * (2 * math.pi / 64)
    X, Y = np.meshgrid(x, x, indexing="ij")
    ref_mean = np.exp(-((X - math.pi) ** 2 + (Y - math.pi) ** 2) / (2 * 0.25)).mean()
    assert abs(float(dye0[0, 0].real) / 64**2 - ref_mean) < 1e-10
    o = load_output(sorted((out / "fields").glob("fields_final_*"))[0])
    assert {"theta", "scalar_dye", "scalar_salt"} <= set(o)
    assert np.allclose(o["scalar_salt"], 2.0, atol=1e-9)
