"""Run configuration and file formats on the host (no GPU): RunConfig
validation and YAML round trip (io/config.py of the reference), the
checkpoint layout (theta_hat_real / theta_hat_imag, time / step attributes,
JSON config), diagnostics time series and field output, and a dry run of
the driver."""

import json
import math

import numpy as np
import pytest
import torch
import yaml

from pygsquig_b200.io import (
    RunConfig,
    load_checkpoint,
    load_config,
    load_diagnostics,
    load_output,
    save_checkpoint,
    save_diagnostics,
    save_output,
)
from pygsquig_b200.io.config import (
    DampingConfig,
    DissipationConfig,
    ForcingConfig,
    GridConfig,
    InitialConditionConfig,
    OutputConfig,
    PassiveScalarConfig,
    ScalarsConfig,
    SimulationConfig,
    SolverConfig,
    TimeIntegrationConfig,
)

CFG = {
    "grid": {"N": 64, "L": 2 * math.pi},
    "solver": {"alpha": 1.0, "dissipation": {"nu_p": 1e-12, "p": 8},
               "damping": {"type": "linear_drag", "mu": 0.1},
               "time_integration": {"dt": 0.002, "adaptive_cfl": False}},
    "forcing": {"type": "ring", "kf": 8.0, "dk": 1.0, "epsilon": 0.1, "seed": 7},
    "simulation": {"t_end": 0.1, "output_interval": 0.05, "checkpoint_interval": 0.05, "log_interval": 0.02},
    "initial_condition": {"type": "random", "seed": 3},
    "output": {"fields": ["theta", "velocity"], "diagnostics": ["energy_spectrum"]},
    "scalars": {"enabled": True, "species": [{"name": "dye", "kappa": 1e-3, "initial_condition": "gaussian",
                                              "initial_params": {"width": 0.5}}]},
}


@pytest.mark.parametrize("make", [
    lambda: GridConfig(N=63), lambda: GridConfig(L=0), lambda: DissipationConfig(p=3),
    lambda: DissipationConfig(type="x"), lambda: DissipationConfig(nu_p=-1), lambda: DampingConfig(mu=-1),
    lambda: DampingConfig(k_cutoff_factor=0), lambda: TimeIntegrationConfig(method="Euler"),
    lambda: TimeIntegrationConfig(dt=0), lambda: TimeIntegrationConfig(cfl_safety=1.0),
    lambda: TimeIntegrationConfig(dt_max=0), lambda: SolverConfig(alpha=2.5), lambda: ForcingConfig(kf=0),
    lambda: ForcingConfig(type="x"), lambda: ForcingConfig(tau_f=-1), lambda: OutputConfig(fields=["rho"]),
    lambda: OutputConfig(diagnostics=["x"]), lambda: SimulationConfig(t_end=0),
    lambda: SimulationConfig(t_end=1, log_interval=0), lambda: PassiveScalarConfig(name="a", kappa=-1),
    lambda: PassiveScalarConfig(name="a", initial_condition="x"),
    lambda: ScalarsConfig(species=[PassiveScalarConfig(name="a"), PassiveScalarConfig(name="a")]),
    lambda: InitialConditionConfig(type="checkpoint"), lambda: InitialConditionConfig(amplitude=0),
])
def test_validation(make):
    with pytest.raises(ValueError):
        make()


def test_yaml_round_trip(tmp_path):
    p = tmp_path / "c.yml"
    p.write_text(yaml.safe_dump(CFG))
    c = load_config(p)
    assert c.grid.N == 64 and c.solver.alpha == 1.0 and c.solver.time_integration.dt == 0.002
    assert c.forcing.seed == 7 and c.scalars.species[0].name == "dye"
    assert c.solver.damping.k_cutoff_factor == 0.5 and c.solver.dissipation.type == "hyperviscosity"
    c.to_yaml(tmp_path / "d.yml")
    c2 = load_config(tmp_path / "d.yml")
    assert c2 == c
    d = c.to_dict()
    assert "wall_time_limit" not in d["simulation"] and "dt_max" not in d["solver"]["time_integration"]
    assert RunConfig.from_dict(json.loads(json.dumps(d))) == c


def test_defaults():
    c = RunConfig.from_dict({"grid": {}, "solver": {"alpha": 0.5}})
    assert c.grid.N == 256 and c.forcing is None and c.scalars is None
    assert c.simulation.t_end == 100.0 and c.solver.time_integration.adaptive_cfl is True
    assert c.output.fields == ["theta"] and c.initial_condition.type == "random"


def test_checkpoint_layout_and_round_trip(tmp_path):
    from pygsquig_b200.scalars.state import MultiScalarState

    c = RunConfig.from_dict(CFG)
    rng = np.random.default_rng(0)
    th = torch.as_tensor(rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64)))
    sh = torch.as_tensor(rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))).to(torch.complex64)
    state = {"theta_hat": th, "time": 1.25, "step": 625, "note": "x", "aux": np.arange(3.0),
             "scalar_state": MultiScalarState(scalars={"dye": sh}, time=1.25, diagnostics={})}
    f = tmp_path / "ck" / "step_00000625.npz"
    save_checkpoint(state, c, f)
    with np.load(f) as z:
        keys = set(z.files)
        assert {"state/theta_hat_real", "state/theta_hat_imag", "state/.attrs", "metadata/.attrs",
                "state/aux", "scalar_state/dye_real", "scalar_state/dye_imag"} <= keys
        meta = json.loads(str(z["metadata/.attrs"]))
        assert {"timestamp", "pygsquig_version", "git_commit", "git_dirty", "config"} <= set(meta)
        assert json.loads(str(z["state/.attrs"])) == {"time": 1.25, "step": 625, "note": "x"}
    st, c2 = load_checkpoint(f)
    assert c2 == c
    assert torch.equal(st["theta_hat"], th) and st["time"] == 1.25 and st["step"] == 625 and st["note"] == "x"
    assert torch.equal(st["scalar_state"].scalars["dye"], sh)
    assert np.array_equal(st["aux"].numpy(), np.arange(3.0))
    save_checkpoint({"theta_hat": th.to(torch.complex64), "time": 0.0, "step": 0}, c, tmp_path / "raw.npz",
                    compression=None)
    st, _ = load_checkpoint(tmp_path / "raw.npz")
    assert st["theta_hat"].dtype == torch.complex64


def test_hdf5_name_needs_h5py(tmp_path):
    from pygsquig_b200.io import checkpoint as ck

    if ck.h5py is not None:
        pytest.skip("h5py installed")
    with pytest.raises(ImportError, match="h5py"):
        save_checkpoint({"theta_hat": torch.zeros(8, 8, dtype=torch.complex128), "time": 0.0, "step": 0},
                        RunConfig.from_dict(CFG), tmp_path / "a.h5")


def test_diagnostics_series(tmp_path):
    f = tmp_path / "ts.npz"
    for t in (0.0, 0.1, 0.1 + 1e-12, 0.2):  # a repeated time is skipped
        save_diagnostics({"energy": 1.0 + t, "spectrum": np.full(4, t)}, t, f)
    d = load_diagnostics(f)
    assert np.allclose(d["time"], [0.0, 0.1, 0.2]) and d["spectrum"].shape == (3, 4)
    assert np.allclose(d["energy"], [1.0, 1.1, 1.2])
    save_diagnostics({"energy": 5.0}, 9.0, f, mode="write")
    assert load_diagnostics(f)["time"].tolist() == [9.0]


def test_output_file(tmp_path):
    from pygsquig_b200.core.grid import Grid  # noqa: F401  (the grid type the writer takes)

    class G:
        N, L = 16, 2 * math.pi

    f = tmp_path / "fields_00000001.npz"
    save_output({"theta": np.ones((16, 16)), "spec": np.zeros((16, 9))}, G, 0.5, {"step": 1, "flag": True}, f)
    o = load_output(f)
    assert o["theta"].shape == (16, 16) and "spec_hat" in o and float(o["time"]) == 0.5
    assert o["attrs"]["N"] == 16 and o["attrs"]["flag"] == "True" and o["x"][1] == pytest.approx(2 * math.pi / 16)


def test_driver_dry_run(tmp_path):
    from pygsquig_b200.run import run

    p = tmp_path / "c.yml"
    p.write_text(yaml.safe_dump(CFG))
    assert run(str(p), output_dir=str(tmp_path / "out"), dry_run=True) is None
    assert not (tmp_path / "out").exists()
