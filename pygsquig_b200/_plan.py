"""Owning wrapper around one libsqg plan and its device workspace."""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


@dataclass(frozen=True)
class PlanKey:
    """Everything a plan depends on (used to cache plans)."""

    N: int
    L: float
    alpha: float
    nu_p: float
    p: int
    precision: str = "float64"
    scheme: str = "explicit"
    damping: Optional[tuple] = None  # (mu, kf, nu_p, p)
    ring: Optional[tuple] = None  # (kf, dk, epsilon, tau_f, amplitude)
    scalars: tuple = field(default_factory=tuple)  # ((kappa, mean_grad, gx, gy), ...)
    role: str = "step"  # "aux": transforms/diagnostics, own workspace (safe to call mid-step)


class Plan:
    """A libsqg plan with a torch-owned workspace on the current CUDA device."""

    def __init__(self, key: PlanKey, device=None):
        lib = _lib.load()
        if not torch.cuda.is_available():
            raise RuntimeError("pygsquig_b200 needs a CUDA device (no CPU fallback)")
        self.key = key
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        d = _lib.SqgDesc()
        d.N = key.N
        d.precision = _lib.SQG_F64 if key.precision == "float64" else _lib.SQG_F32
        d.scheme = _lib.SQG_EXPLICIT_RK4 if key.scheme == "explicit" else _lib.SQG_IF_RK4
        d.p = int(key.p)
        d.L = float(key.L)
        d.alpha = float(key.alpha)
        d.nu_p = float(key.nu_p)
        if key.damping is not None:
            mu, kf, nu_d, p_d = key.damping
            d.has_damping, d.mu, d.kf_damp, d.nu_damp, d.p_damp = 1, mu, kf, nu_d, int(p_d)
        else:
            d.p_damp = 8
        if key.ring is not None:
            kf, dk, eps, tau, amp = key.ring
            d.has_ring, d.ring_kf, d.ring_dk, d.ring_epsilon, d.ring_tau_f, d.ring_amplitude = 1, kf, dk, eps, tau, amp
        d.n_scalars = len(key.scalars)
        for i, (kappa, mg, gx, gy) in enumerate(key.scalars):
            d.kappa[i] = kappa
            d.mean_gradient[i] = 1 if mg else 0
            d.grad_x[i] = gx
            d.grad_y[i] = gy
        self._desc = d
        h = C.c_void_p()
        _lib.check(lib.sqg_plan_create(C.byref(d), C.byref(h)))
        self._h = h
        self._lib = lib
        nbytes = C.c_size_t()
        _lib.check(lib.sqg_plan_workspace_bytes(h, C.byref(nbytes)))
        self.ws_bytes = int(nbytes.value)
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(self.ws_bytes + 256, dtype=torch.uint8, device=self.device)
            base = self.workspace.data_ptr()
            off = (-base) % 256
            self._ws_off = off
            _lib.check(lib.sqg_plan_set_workspace(h, base + off, self.ws_bytes, _stream_ptr()))
        n = C.c_int32()
        _lib.check(lib.sqg_ring_mode_count(h, C.byref(n)))
        self.n_ring = int(n.value)
        self.cdtype = torch.complex128 if key.precision == "float64" else torch.complex64
        self.rdtype = torch.float64 if key.precision == "float64" else torch.float32

    # ---- helpers ----
    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._lib.sqg_plan_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def ring_modes(self):
        n = self.n_ring
        ix = (C.c_int32 * max(n, 1))()
        iy = (C.c_int32 * max(n, 1))()
        _lib.check(self._lib.sqg_ring_modes(self._h, ix, iy))
        return np.array(ix[:n], dtype=np.int64), np.array(iy[:n], dtype=np.int64)

    def buffer(self, which: int, dtype, shape) -> torch.Tensor:
        off, nb = C.c_size_t(), C.c_size_t()
        _lib.check(self._lib.sqg_plan_buffer(self._h, which, C.byref(off), C.byref(nb)))
        start = self._ws_off + int(off.value)
        el = torch.empty((), dtype=dtype).element_size()
        count = int(np.prod(shape))
        return self.workspace[start : start + count * el].view(dtype).view(*shape)

    def host_tables(self):
        N = self.key.N
        k = (C.c_double * N)()
        dm = (C.c_int32 * N)()
        dr = (C.c_int32 * N)()
        _lib.check(self._lib.sqg_plan_host_tables(self._h, k, dm, dr))
        return np.array(k[:]), np.array(dm[:]), np.array(dr[:])

    def check_spectrum(self, t: torch.Tensor, name="theta_hat") -> torch.Tensor:
        N = self.key.N
        if not isinstance(t, torch.Tensor):
            t = torch.as_tensor(np.asarray(t))
        if t.shape != (N, N):
            raise ValueError(f"{name} must have shape ({N}, {N}), got {tuple(t.shape)}")
        if not t.is_complex():
            t = t.to(torch.float64)
        return t.to(device=self.device, dtype=self.cdtype).contiguous()

    def check_real(self, t, name="field") -> torch.Tensor:
        N = self.key.N
        if not isinstance(t, torch.Tensor):
            t = torch.as_tensor(np.asarray(t, dtype=np.float64))
        if t.shape != (N, N):
            raise ValueError(f"{name} must have shape ({N}, {N}), got {tuple(t.shape)}")
        return t.to(device=self.device, dtype=self.rdtype).contiguous()

    def phases_tensor(self, key, n_steps: Optional[int] = None) -> Optional[torch.Tensor]:
        """Host-drawn ring phases -> device float64 [n_ring] (or [n_steps, n_ring]).

        Accepts the ring-ordered 1-D phases, or a full (N, N) phase array as
        the reference's ``_generate_random_phases`` returns (ring_forcing.py:
        78-92), from which the ring entries are gathered.
        """
        if self.n_ring == 0:
            return None
        if key is None:
            raise ValueError("ring forcing needs host-drawn phases (the `key` argument)")
        t = key if isinstance(key, torch.Tensor) else torch.as_tensor(np.asarray(key, dtype=np.float64))
        t = t.to(device=self.device, dtype=torch.float64)
        N = self.key.N
        if n_steps is None:
            if t.dim() == 2 and t.shape == (N, N):
                ix, iy = self.ring_modes()
                t = t[torch.as_tensor(ix, device=self.device), torch.as_tensor(iy, device=self.device)]
            if t.shape != (self.n_ring,):
                raise ValueError(f"phases must have shape ({self.n_ring},) or ({N}, {N})")
        else:
            if t.shape != (n_steps, self.n_ring):
                raise ValueError(f"noise must have shape ({n_steps}, {self.n_ring})")
        return t.contiguous()

    # ---- calls ----
    def rhs(self, th, out=None):
        if out is None:
            out = torch.empty_like(th)
        _lib.check(self._lib.sqg_rhs(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out

    def step(self, th_in, th_out, dt, phases=None):
        _lib.check(self._lib.sqg_step(self._h, th_in.data_ptr(), th_out.data_ptr(), float(dt), _ptr(phases), _stream_ptr()))

    def multistep(self, th, n, dt, phases=None, use_graph=True):
        _lib.check(
            self._lib.sqg_multistep(self._h, th.data_ptr(), int(n), float(dt), _ptr(phases), 1 if use_graph else 0,
                                    _stream_ptr())
        )

    def stage_begin(self, th_in):
        _lib.check(self._lib.sqg_stage_begin(self._h, th_in.data_ptr(), _stream_ptr()))

    def stage(self, s, th_in, th_out, dt, extra=None, phases=None):
        _lib.check(self._lib.sqg_stage(self._h, int(s), th_in.data_ptr(), th_out.data_ptr(), float(dt), _ptr(extra),
                                       _ptr(phases), _stream_ptr()))

    def stage_physical(self, s, th_in, th_out, dt, src, phases=None):
        """Stage s with a physical-space tendency ``src`` (real N x N, plan
        precision) added to the advective term and dealiased with it."""
        _lib.check(self._lib.sqg_stage_physical(self._h, int(s), th_in.data_ptr(), th_out.data_ptr(), float(dt),
                                                src.data_ptr(), _ptr(phases), _stream_ptr()))

    def velocity(self, th):
        N = self.key.N
        u = torch.empty((N, N), dtype=self.rdtype, device=self.device)
        v = torch.empty_like(u)
        _lib.check(self._lib.sqg_velocity(self._h, th.data_ptr(), u.data_ptr(), v.data_ptr(), _stream_ptr()))
        return u, v

    def to_physical(self, fh, out=None):
        N = self.key.N
        if out is None:
            out = torch.empty((N, N), dtype=self.rdtype, device=self.device)
        _lib.check(self._lib.sqg_to_physical(self._h, fh.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out

    def to_spectral(self, f, out=None):
        N = self.key.N
        if out is None:
            out = torch.empty((N, N), dtype=self.cdtype, device=self.device)
        _lib.check(self._lib.sqg_to_spectral(self._h, f.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out

    def damping(self, th):
        out = torch.empty_like(th)
        _lib.check(self._lib.sqg_damping(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out

    def hyperviscosity(self, th):
        out = torch.empty_like(th)
        _lib.check(self._lib.sqg_hyperviscosity(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out

    def ring_forcing(self, th, phases, dt):
        out = torch.empty_like(th)
        _lib.check(self._lib.sqg_ring_forcing(self._h, th.data_ptr(), _ptr(phases), float(dt), out.data_ptr(),
                                              _stream_ptr()))
        return out

    def inner(self, a, b) -> float:
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_inner(self._h, a.data_ptr(), b.data_ptr(), out.data_ptr(), _stream_ptr()))
        return float(out.item())

    def diagnostics(self, th) -> np.ndarray:
        out = torch.empty(_lib.SQG_DIAG_COUNT, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_diagnostics(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out.cpu().numpy()

    def energy_spectrum(self, th) -> np.ndarray:
        nb = min(self.key.N // 4, 64)
        out = torch.empty(nb, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_energy_spectrum(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return out.cpu().numpy()

    def max_speed(self, u, v) -> float:
        """max sqrt(u^2 + v^2) (NaN if a value is not finite)."""
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_max_speed(self._h, u.data_ptr(), v.data_ptr(), out.data_ptr(), _stream_ptr()))
        return float(out.item())

    def spectrum_absmax(self, th) -> float:
        """max |theta_hat| (NaN if a value is not finite)."""
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_spectrum_absmax(self._h, th.data_ptr(), out.data_ptr(), _stream_ptr()))
        return float(out.item())

    def scalar_variance(self, sh) -> float:
        out = torch.empty(1, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.sqg_scalar_variance(self._h, sh.data_ptr(), out.data_ptr(), _stream_ptr()))
        return float(out.item())

    def scalars_step(self, th_new, s_in: Sequence[torch.Tensor], s_out: Sequence[torch.Tensor], dt):
        n = len(s_in)
        arr_in = (C.c_void_p * max(n, 1))(*[t.data_ptr() for t in s_in])
        arr_out = (C.c_void_p * max(n, 1))(*[t.data_ptr() for t in s_out])
        _lib.check(self._lib.sqg_scalars_step(self._h, th_new.data_ptr(), arr_in, arr_out, float(dt), _stream_ptr()))

    def ring_substeps(self, th, n_sub, dt_sub, phases):
        """n_sub forcing-only RK4 sub-steps on the ring modes of th (in place);
        phases: device float64 [n_sub, n_ring]."""
        _lib.check(self._lib.sqg_ring_substeps(self._h, th.data_ptr(), int(n_sub), float(dt_sub), _ptr(phases),
                                               _stream_ptr()))

    # ---- launch shapes ----
    def shape(self) -> dict:
        """Current and maximal launch shapes: row pairs per CTA of the row
        pass (rpc) and column pairs per CTA of the column pass (np)."""
        v = [C.c_int32() for _ in range(4)]
        _lib.check(self._lib.sqg_plan_shape(self._h, *[C.byref(x) for x in v]))
        return {"rpc": v[0].value, "np": v[1].value, "max_rpc": v[2].value, "max_np": v[3].value}

    def set_shape(self, rpc: int = 0, np_: int = 0) -> None:
        """Select launch shapes (0: the compiled maximum).  Results are
        bit-identical for every shape."""
        _lib.check(self._lib.sqg_plan_set_shape(self._h, int(rpc), int(np_)))

    def autotune(self, reps: int = 5) -> dict:
        """Time every launch shape on this plan's workspace and keep the
        fastest (synchronises the current stream)."""
        _lib.check(self._lib.sqg_plan_autotune(self._h, int(reps), _stream_ptr()))
        return self.shape()

    def check_status(self) -> int:
        """Reads and clears the plan's status flags; returns bit 0 (non-finite
        value seen).  Bit 1 (a column pass's tile copies did not complete
        within the wait limit) raises."""
        f = C.c_uint32()
        _lib.check(self._lib.sqg_check_status(self._h, C.byref(f), _stream_ptr()))
        if int(f.value) & 2:
            raise RuntimeError("column pass: TMA tile copies did not complete within the wait limit")
        return int(f.value) & 1

    TIMING_KINDS = ("row_inverse", "row_stage", "col_theta", "row_scalar", "col_scalar", "other", "row_last",
                    "row_vel", "col_vel", "row_scalar_inverse")

    def set_timing(self, on, reps: int = 1) -> None:
        """on=False: off.  on=True: events around every launch site, each site
        issuing ``reps`` launches of its pass back to back (reps > 1: the
        results of the timed calls are not valid)."""
        _lib.check(self._lib.sqg_set_timing(self._h, (max(int(reps), 1)) if on else 0))

    def timing_read(self) -> dict:
        n = len(self.TIMING_KINDS)
        ms = (C.c_double * n)()
        cnt = (C.c_int64 * n)()
        _lib.check(self._lib.sqg_timing_read(self._h, ms, cnt, n))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(self.TIMING_KINDS)}

    def last_launch_count(self) -> int:
        n = C.c_int64()
        _lib.check(self._lib.sqg_last_launch_count(self._h, C.byref(n)))
        return int(n.value)


_CACHE: dict = {}

# Plans pick their launch shapes by timing them when they are created.
AUTOTUNE = True


def get_plan(key: PlanKey) -> Plan:
    dev = torch.cuda.current_device() if torch.cuda.is_available() else -1
    k = (key, dev)
    pl = _CACHE.get(k)
    if pl is None:
        pl = Plan(key)
        if AUTOTUNE:
            pl.autotune()
        _CACHE[k] = pl
    return pl


_GENERATION = [0]


def plan_generation() -> int:
    """Incremented by clear_plans (callers that keep plans drop them then)."""
    return _GENERATION[0]


def clear_plans() -> None:
    _CACHE.clear()
    _GENERATION[0] += 1
