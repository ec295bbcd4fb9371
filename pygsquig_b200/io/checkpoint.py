"""Checkpoints, field output and diagnostics time series (mirrors
pygsquig/io/hdf5_io.py).

The layout is the reference's: group ``metadata`` with attributes
``timestamp``, ``pygsquig_version``, ``git_commit``, ``git_dirty``
(``git_status``) and ``config`` (the run configuration as JSON); group
``state`` with datasets ``theta_hat_real`` / ``theta_hat_imag`` and
attributes ``time`` / ``step``; extra arrays as ``<key>`` or
``<key>_real`` / ``<key>_imag``, extra scalars as attributes.

Two containers hold that layout.  HDF5 (``.h5`` / ``.hdf5`` names) needs
h5py and is written exactly like the reference's file, so either program
can resume from the other's checkpoints.  Every other name is a NumPy
``.npz`` archive whose keys are the HDF5 paths (``state/theta_hat_real``)
and whose attributes are JSON under ``<group>/.attrs``.  Passive scalars of
a ``gSQGSolverWithScalars`` state are stored under ``scalar_state/<name>``.
"""

from __future__ import annotations

import io
import json
import os
import subprocess
from datetime import datetime
from pathlib import Path
from typing import Any, Union

import numpy as np
import torch

from .config import RunConfig

try:  # optional: HDF5 containers
    import h5py  # type: ignore
except ImportError:  # pragma: no cover - depends on the environment
    h5py = None

VERSION = "0.1.0"


def _np(x) -> np.ndarray:
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def _git_info() -> dict:
    """Commit and dirty flag of the working directory (hdf5_io.py:22-46)."""
    try:
        commit = subprocess.check_output(["git", "rev-parse", "HEAD"], stderr=subprocess.DEVNULL).decode().strip()
        status = subprocess.check_output(["git", "status", "--porcelain"], stderr=subprocess.DEVNULL).decode().strip()
        return {"commit": commit, "dirty": bool(status), "status": status[:1000] if status else ""}
    except (subprocess.CalledProcessError, FileNotFoundError, OSError):
        return {"commit": "unknown", "dirty": False, "status": ""}


def _is_hdf5(path: Path) -> bool:
    return path.suffix.lower() in (".h5", ".hdf5")


def _need_h5py(path: Path):
    if h5py is None:
        raise ImportError(f"{path}: HDF5 files need h5py, which is not installed; use a .npz file name")


class _Tree:
    """Groups of arrays and attributes, written to HDF5 or to an npz archive."""

    def __init__(self):
        self.arrays: dict[str, np.ndarray] = {}
        self.attrs: dict[str, dict] = {}

    def write(self, path: Path, compress: bool = True, level: int = 4):
        path.parent.mkdir(parents=True, exist_ok=True)
        if _is_hdf5(path):
            _need_h5py(path)
            with h5py.File(path, "w") as f:
                for key, arr in self.arrays.items():
                    kw = dict(compression="gzip", compression_opts=level) if compress and arr.ndim else {}
                    f.create_dataset(key, data=arr, **kw)
                for grp, attrs in self.attrs.items():
                    obj = f.require_group(grp) if grp else f
                    for k, v in attrs.items():
                        obj.attrs[k] = v
            return
        payload = dict(self.arrays)
        for grp, attrs in self.attrs.items():
            payload[f"{grp}/.attrs"] = np.array(json.dumps(attrs))
        buf = io.BytesIO()
        (np.savez_compressed if compress else np.savez)(buf, **payload)
        tmp = path.with_name(path.name + ".tmp")
        with open(tmp, "wb") as f:
            f.write(buf.getvalue())
        os.replace(tmp, path)  # a reader never sees a half-written file

    @classmethod
    def read(cls, path: Path) -> "_Tree":
        t = cls()
        if _is_hdf5(path):
            _need_h5py(path)
            with h5py.File(path, "r") as f:
                def visit(name, obj):
                    if isinstance(obj, h5py.Dataset):
                        t.arrays[name] = obj[()]
                    else:
                        t.attrs[name] = {k: _plain(v) for k, v in obj.attrs.items()}
                f.visititems(visit)
                t.attrs[""] = {k: _plain(v) for k, v in f.attrs.items()}
            return t
        with np.load(path, allow_pickle=False) as z:
            for key in z.files:
                if key.endswith("/.attrs"):
                    t.attrs[key[: -len("/.attrs")]] = json.loads(str(z[key]))
                else:
                    t.arrays[key] = z[key]
        return t


def _plain(v):
    if isinstance(v, bytes):
        return v.decode()
    if isinstance(v, np.generic):
        return v.item()
    return v


def _put_array(tree: _Tree, key: str, arr: np.ndarray):
    if np.iscomplexobj(arr):
        tree.arrays[f"{key}_real"] = np.ascontiguousarray(arr.real)
        tree.arrays[f"{key}_imag"] = np.ascontiguousarray(arr.imag)
    else:
        tree.arrays[key] = arr


def save_checkpoint(state: dict[str, Any], config: RunConfig, filename: Union[str, Path],
                    compression: str = "gzip", compression_level: int = 4) -> None:
    """hdf5_io.py:49-123.  ``compression=None`` stores the arrays raw."""
    path = Path(filename)
    tree = _Tree()
    git = _git_info()
    meta = {"timestamp": datetime.now().isoformat(), "pygsquig_version": VERSION,
            "git_commit": git["commit"], "git_dirty": git["dirty"],
            "config": json.dumps(config.to_dict())}
    if git["dirty"]:
        meta["git_status"] = git["status"]
    tree.attrs["metadata"] = meta
    th = _np(state["theta_hat"])
    tree.arrays["state/theta_hat_real"] = np.ascontiguousarray(th.real)
    tree.arrays["state/theta_hat_imag"] = np.ascontiguousarray(th.imag)
    sattrs = {"time": float(state["time"]), "step": int(state["step"])}
    for key, value in state.items():
        if key in ("theta_hat", "time", "step"):
            continue
        if key == "scalar_state" and value is not None:
            scal = value.scalars if hasattr(value, "scalars") else value.get("scalars", {})
            for name, sh in scal.items():
                _put_array(tree, f"scalar_state/{name}", _np(sh))
        elif isinstance(value, (np.ndarray, torch.Tensor)):
            _put_array(tree, f"state/{key}", _np(value))
        elif isinstance(value, (bool, int, float, str)):
            sattrs[key] = value
    tree.attrs["state"] = sattrs
    tree.write(path, compress=compression is not None, level=compression_level)


def _complex_pairs(arrays: dict, prefix: str) -> dict:
    out = {}
    for key, arr in arrays.items():
        if not key.startswith(prefix):
            continue
        name = key[len(prefix):]
        if name.endswith("_real") and f"{prefix}{name[:-5]}_imag" in arrays:
            im = arrays[f"{prefix}{name[:-5]}_imag"]
            out[name[:-5]] = torch.complex(torch.as_tensor(arr), torch.as_tensor(im))
        elif not name.endswith("_imag"):
            out[name] = torch.as_tensor(arr)
    return out


def load_checkpoint(filename: Union[str, Path]) -> tuple[dict[str, Any], RunConfig]:
    """hdf5_io.py:126-178: (state, config).  Arrays come back as CPU torch
    tensors (the solvers move them to their device)."""
    tree = _Tree.read(Path(filename))
    config = RunConfig.from_dict(json.loads(tree.attrs["metadata"]["config"]))
    fields = _complex_pairs(tree.arrays, "state/")
    sattrs = tree.attrs.get("state", {})
    state: dict[str, Any] = {"theta_hat": fields.pop("theta_hat"), "time": float(sattrs["time"]),
                             "step": int(sattrs["step"])}
    state.update(fields)
    for k, v in sattrs.items():
        if k not in ("time", "step"):
            state[k] = v
    scal = _complex_pairs(tree.arrays, "scalar_state/")
    if scal:
        from ..scalars.state import MultiScalarState

        state["scalar_state"] = MultiScalarState(scalars=scal, time=state["time"], diagnostics={})
    return state, config


def save_output(data: dict, grid, time: float, metadata: dict, filename: Union[str, Path],
                compress: bool = True) -> None:
    """Physical fields with x / y coordinates and attributes (hdf5_io.py:181-256,
    which writes the same through xarray): arrays ``<name>`` with dims (y, x)
    in the reference's ``ifft2(...).real`` layout, ``x``, ``y``, ``time``;
    attributes ``N``, ``L``, ``created`` and the metadata."""
    tree = _Tree()
    N = grid.N
    for name, f in data.items():
        arr = _np(f)
        if arr.shape == (N, N):
            tree.arrays[name] = arr
        elif arr.shape == (N, N // 2 + 1):
            tree.arrays[f"{name}_hat"] = arr
    x = np.arange(N) * (grid.L / N)
    tree.arrays["x"] = x
    tree.arrays["y"] = x.copy()
    tree.arrays["time"] = np.array(float(time))
    attrs = {k: (str(v) if isinstance(v, bool) else v) for k, v in metadata.items()}
    attrs.update(created=datetime.now().isoformat(), N=int(N), L=float(grid.L))
    tree.attrs[""] = attrs
    tree.write(Path(filename), compress=compress)


def load_output(filename: Union[str, Path]) -> dict:
    """Arrays of an output file plus its attributes under ``attrs``."""
    tree = _Tree.read(Path(filename))
    out: dict[str, Any] = dict(tree.arrays)
    out["attrs"] = tree.attrs.get("", {})
    return out


def save_diagnostics(diagnostics: dict, time: float, filename: Union[str, Path], mode: str = "append") -> None:
    """Append one record to a diagnostics time series (hdf5_io.py:271-341):
    ``time`` plus one row per diagnostic; a time already present (np.isclose)
    is not added twice; ``mode="write"`` starts a new series."""
    path = Path(filename)
    rows = {k: np.asarray(_np(v) if isinstance(v, torch.Tensor) else v) for k, v in diagnostics.items()
            if k != "time"}  # the series' own time axis
    if mode == "write" or not path.exists():
        tree = _Tree()
        tree.arrays["time"] = np.array([time], dtype=np.float64)
        for k, v in rows.items():
            tree.arrays[k] = v[np.newaxis, ...]
        tree.write(path, compress=False)
        return
    tree = _Tree.read(path)
    if np.any(np.isclose(tree.arrays["time"], time)):
        return
    n = tree.arrays["time"].shape[0]
    tree.arrays["time"] = np.append(tree.arrays["time"], time)
    for k, v in rows.items():
        if k in tree.arrays and tree.arrays[k].shape[0] == n:
            tree.arrays[k] = np.concatenate([tree.arrays[k], v[np.newaxis, ...]], axis=0)
    tree.write(path, compress=False)


def load_diagnostics(filename: Union[str, Path]) -> dict[str, np.ndarray]:
    """hdf5_io.py:344-359."""
    return dict(_Tree.read(Path(filename)).arrays)
