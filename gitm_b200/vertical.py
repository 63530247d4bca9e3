"""Python host interface of the B200 vertical advance.

Mirrors the reference's entry points for this path, with the module
variables they read made explicit:

=========================  ==============================================
reference                  here
=========================  ==============================================
advance_vertical_all       ``advance_vertical_all(ctx, members, dt)``
(advance_vertical.f90:8)   (device tensors) / ``advance_vertical_all_host``
advance_vertical_1d_*      ``advance_vertical_1d(ctx, columns, dt)``
(vertical_solver_*.f90)    (ModVertical-form device tensors)
calc_timestep_vertical     ``calc_timestep_vertical(ctx, members, ...)``
(calc_timestep.f90:85)
stop_gitm                  ``GitmStop`` (raised instead of aborting)
=========================  ==============================================

State lives in torch tensors on the GPU in the native layout
[field, cell, column] (float64, contiguous).  All compute goes through
libgitmvert.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import abi
from ._lib import lib

# stop_gitm messages of the reference for each status bit
STOP_MESSAGES = {
    abi.ST_NEG_DENSITY: "negative density found! Can't Continue (advance_vertical.f90:96-100)",
    abi.ST_NEG_ION_TOP: "Negative Ion density too close to the upper boundary "
                        "(set_vertical_bcs.Earth.f90:617-620)",
    abi.ST_LU_SINGULAR: "singular matrix in ludcmp (ludcmp.f:11-14)",
    abi.ST_NONFINITE: "NaN or Inf in the vertical solution (check_for_nans.f90)",
    abi.ST_BAD_NALTS: "nAlts outside the range of the launch",
    abi.ST_ADJ_BRANCH: "the adjoint met the upper ion boundary's negative-density repair, which it does "
                       "not differentiate",
    abi.ST_LOW_TEMPERATURE: "Temperature < 100.0 (exchange_messages_sphere.f90:78-82)",
}


class GitmStop(RuntimeError):
    """Raised where the reference would call stop_gitm."""

    def __init__(self, status: int, n_bad: int, detail: str = ""):
        msgs = [m for bit, m in STOP_MESSAGES.items() if status & bit]
        super().__init__(f"{n_bad} column(s) stopped: " + "; ".join(msgs) + (f" [{detail}]" if detail else ""))
        self.status = status
        self.n_bad = n_bad


class GitmError(RuntimeError):
    pass


def _check(rc: int, ctx_handle=None, what: str = ""):
    if rc == abi.OK:
        return
    msg = lib().gitm_vert_last_error(ctx_handle).decode() if ctx_handle else ""
    if rc == abi.ERR_COLUMN:
        raise GitmStop(-1, -1, msg)
    raise GitmError(f"{what} failed with code {rc}: {msg}")


class VerticalContext:
    """A device context with the run-time flags of ModInputs (GitmVertParams)."""

    def __init__(self, params: abi.GitmVertParams | None = None, device: int = 0):
        self.params = params if params is not None else abi.default_params()
        h = C.c_void_p()
        rc = lib().gitm_vert_create(C.byref(self.params), device, C.byref(h))
        if rc != abi.OK:
            raise GitmError(f"gitm_vert_create failed with code {rc} (is a CUDA device visible?)")
        self.handle = h
        self.device = device

    def set_params(self, params: abi.GitmVertParams):
        _check(lib().gitm_vert_set_params(self.handle, C.byref(params)), self.handle, "set_params")
        self.params = params

    def close(self):
        if getattr(self, "handle", None):
            lib().gitm_vert_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return lib().gitm_vert_last_error(self.handle).decode()


# ------------------------------------------------------------------ members
FIELDS = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel", "log_ns",
          "ndensity", "gamma", "mean_major_mass", "temp_unit", "cmax", "ivel_up", "eddy",
          "cos_lat", "sza", "mlat", "lbc", "altitude", "gravity", "dalt_c", "inv_r", "heating",
          "heating_scale")


@dataclasses.dataclass
class DeviceMember:
    """One member's arrays as CUDA float64 tensors (names as GitmColumnBatch)."""

    n_alts: int
    n_cols: int
    tensors: dict

    def batch(self) -> abi.GitmColumnBatch:
        b = abi.GitmColumnBatch()
        b.n_alts = self.n_alts
        b.n_cols = self.n_cols
        alt = self.tensors["altitude"]
        b.grid_per_column = 1 if alt.dim() == 2 else 0
        for name in FIELDS:
            t = self.tensors.get(name)
            if t is None:
                setattr(b, name, abi.dptr(0))
                continue
            if not (t.is_cuda and t.dtype == _torch().float64 and t.is_contiguous()):
                raise GitmError(f"{name}: expected a contiguous float64 CUDA tensor")
            setattr(b, name, abi.dptr(t.data_ptr()))
        return b

    def to_numpy(self) -> dict:
        return {k: v.detach().cpu().numpy() for k, v in self.tensors.items() if v is not None}


def _torch():
    import torch
    return torch


def device_member(m, device="cuda") -> DeviceMember:
    """Copies a synthetic.Member (numpy) to the GPU."""
    torch = _torch()
    ts = {}
    for name in FIELDS:
        a = getattr(m, name, None)
        ts[name] = None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(device)
    return DeviceMember(m.n_alts, m.n_cols, ts)


class _DeviceArray:
    """A raw device allocation exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr,
                                         "data": (int(ptr or 0), False), "version": 3}


def _batch_array(members):
    arr = (abi.GitmColumnBatch * len(members))(*[mm.batch() for mm in members])
    return arr


class Plan:
    """A batch of members prepared once (member table, grid coefficients,
    tile list) and advanced any number of times; ``advance`` only launches
    kernels, so it can be captured in a CUDA graph."""

    def __init__(self, ctx: VerticalContext, members):
        self.ctx = ctx
        self.members = list(members)
        self._arr = _batch_array(self.members)
        h = C.c_void_p()
        _check(lib().gitm_vert_plan_create(ctx.handle, self._arr, len(self.members), C.byref(h)),
               ctx.handle, "plan_create")
        self.handle = h

    @property
    def config(self) -> abi.GitmLaunchConfig:
        c = abi.GitmLaunchConfig()
        _check(lib().gitm_vert_plan_get_config(self.handle, C.byref(c)), self.ctx.handle)
        return c

    def set_config(self, threads=256, cols_per_cta=0, steps_per_launch=1, ctas_per_sm=0):
        c = abi.GitmLaunchConfig(threads, cols_per_cta, steps_per_launch, ctas_per_sm)
        _check(lib().gitm_vert_plan_set_config(self.handle, C.byref(c)), self.ctx.handle, "set_config")

    def advance(self, dt: float, n_steps: int = 1, stream=None):
        s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
        _check(lib().gitm_vert_plan_advance(self.handle, dt, n_steps, C.c_void_p(s)),
               self.ctx.handle, "plan_advance")

    def saved_state_doubles(self) -> int:
        """Doubles of the buffer advance_saving fills."""
        return int(lib().gitm_vert_plan_saved_state_doubles(self.handle))

    def advance_saving(self, dt: float, states, stream=None):
        """gitm_vert_plan_advance_saving: one step that also saves its stage
        states (a float64 CUDA tensor of saved_state_doubles() elements)."""
        torch = _torch()
        if not (states.is_cuda and states.dtype == torch.float64 and states.is_contiguous()
                and states.numel() >= self.saved_state_doubles()):
            raise GitmError("states: expected a contiguous float64 CUDA tensor of saved_state_doubles() elements")
        s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
        _check(lib().gitm_vert_plan_advance_saving(self.handle, dt, C.c_void_p(states.data_ptr()), C.c_void_p(s)),
               self.ctx.handle, "plan_advance_saving")

    def adjoint(self, bars, dt: float, saved=None, stream=None):
        """gitm_vert_plan_adjoint: bars is one dict per member of adjoint
        tensors named like the GitmColumnAdjoint fields (state arrays in:
        ybar, out: xbar; eddy / heating_scale accumulate).  saved: the
        buffer advance_saving filled for this step, or None."""
        bars = list(bars) if isinstance(bars, (list, tuple)) else [bars]
        arr = (abi.GitmColumnAdjoint * len(bars))()
        torch = _torch()
        for a, d in zip(arr, bars):
            for name, _ in abi.GitmColumnAdjoint._fields_:
                t = d.get(name)
                if t is None:
                    setattr(a, name, abi.dptr(0))
                    continue
                if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                    raise GitmError(f"{name}: expected a contiguous float64 CUDA tensor")
                setattr(a, name, abi.dptr(t.data_ptr()))
        s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
        sp = 0 if saved is None else saved.data_ptr()
        _check(lib().gitm_vert_plan_adjoint(self.handle, arr, dt, C.c_void_p(sp), C.c_void_p(s)), self.ctx.handle,
               "plan_adjoint")

    def autotune(self, dt: float, n_steps: int = 1) -> abi.GitmLaunchConfig:
        c = abi.GitmLaunchConfig()
        _check(lib().gitm_vert_plan_autotune(self.handle, dt, n_steps, C.byref(c)), self.ctx.handle,
               "autotune")
        return c

    def launch_count(self, n_steps: int) -> int:
        return lib().gitm_vert_plan_launch_count(self.handle, n_steps)

    def status(self, clear: bool = False):
        st = C.c_uint32()
        nb = C.c_int64()
        _check(lib().gitm_vert_plan_status(self.handle, C.byref(st), C.byref(nb), int(clear)),
               self.ctx.handle, "plan_status")
        return st.value, nb.value

    def wait(self, timeout_s: float, stream=None) -> bool:
        """gitm_vert_plan_wait: True once the work issued on `stream` has
        finished, False when timeout_s passed first (the work still runs)."""
        s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
        rc = lib().gitm_vert_plan_wait(self.handle, C.c_void_p(s), float(timeout_s))
        if rc == abi.ERR_TIMEOUT:
            return False
        _check(rc, self.ctx.handle, "plan_wait")
        return True

    def check(self, clear: bool = True):
        st, nb = self.status(clear)
        if st:
            raise GitmStop(st, nb)

    def status_words(self):
        """Per-column status words as a numpy uint32 array (synchronises)."""
        torch = _torch()
        n = sum(m.n_cols for m in self.members)
        ptr = lib().gitm_vert_plan_status_words(self.handle)
        view = _DeviceArray(ptr, n, "<i4")
        torch.cuda.synchronize()
        t = torch.as_tensor(view, device=f"cuda:{self.ctx.device}")
        return t.cpu().numpy().view(np.uint32).copy()

    def close(self):
        if getattr(self, "handle", None):
            lib().gitm_vert_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ one-shot calls
def advance_vertical_all(ctx: VerticalContext, members, dt: float, n_steps: int = 1):
    """advance_vertical_all on device tensors: one plan, n_steps, synchronised;
    raises GitmStop where the reference would stop."""
    members = list(members) if isinstance(members, (list, tuple)) else [members]
    arr = _batch_array(members)
    rc = lib().gitm_vert_advance_native(ctx.handle, arr, len(members), dt, n_steps)
    if rc == abi.ERR_COLUMN:
        raise GitmStop(-1, -1, ctx.last_error())
    _check(rc, ctx.handle, "advance_native")


def host_batch(m) -> abi.GitmColumnBatch:
    """GitmColumnBatch of host numpy arrays (synthetic.Member)."""
    b = abi.GitmColumnBatch()
    b.n_alts = m.n_alts
    b.n_cols = m.n_cols
    b.grid_per_column = 1 if np.ndim(m.altitude) == 2 else 0
    for name in FIELDS:
        a = getattr(m, name, None)
        if a is None:
            setattr(b, name, abi.dptr(0))
            continue
        assert a.dtype == np.float64 and a.flags.c_contiguous, name
        setattr(b, name, abi.dptr(a.ctypes.data))
    return b


def advance_vertical_all_host(ctx: VerticalContext, members, dt: float, n_steps: int = 1):
    """advance_vertical_all on host numpy arrays (copied in and out)."""
    members = list(members) if isinstance(members, (list, tuple)) else [members]
    arr = (abi.GitmColumnBatch * len(members))(*[host_batch(m) for m in members])
    rc = lib().gitm_vert_advance_native_host(ctx.handle, arr, len(members), dt, n_steps)
    if rc == abi.ERR_COLUMN:
        raise GitmStop(-1, -1, ctx.last_error())
    _check(rc, ctx.handle, "advance_native_host")


MODVERT_FIELDS = ("log_rho", "temp", "vel_gd", "log_ns", "vert_vel", "log_ins", "ivel", "cmax",
                  "mean_major_mass", "gamma", "eddy", "centrifugal", "coriolis", "sza", "mlat",
                  "lbc", "altitude", "gravity", "dalt_c", "inv_r", "heating", "heating_scale")


def advance_vertical_1d(ctx: VerticalContext, cols: dict, dt: float):
    """One RK4 step of advance_vertical_1d_rusanov on ModVertical-form device
    tensors (dict with MODVERT_FIELDS, updated in place)."""
    torch = _torch()
    b = abi.GitmModVerticalBatch()
    b.n_alts = int(cols["n_alts"])
    b.n_cols = int(cols["n_cols"])
    b.grid_per_column = 1 if cols["altitude"].dim() == 2 else 0
    for name in MODVERT_FIELDS:
        t = cols.get(name)
        if t is None:
            setattr(b, name, abi.dptr(0))
            continue
        assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous(), name
        setattr(b, name, abi.dptr(t.data_ptr()))
    rc = lib().gitm_vert_advance_1d(ctx.handle, C.byref(b), dt, None)
    if rc == abi.ERR_COLUMN:
        raise GitmStop(-1, -1, ctx.last_error())
    _check(rc, ctx.handle, "advance_1d")


def calc_timestep_vertical(ctx: VerticalContext, members, cfl: float = 0.75, dt: float = 1.0e32,
                           dt_end: float = 1.0e32) -> float:
    """calc_timestep_vertical: writes cMax and returns min(dt, CFL step, dt_end)."""
    members = list(members) if isinstance(members, (list, tuple)) else [members]
    arr = _batch_array(members)
    out = C.c_double()
    _check(lib().gitm_vert_cfl_dt(ctx.handle, arr, len(members), cfl, dt, dt_end, C.byref(out)),
           ctx.handle, "cfl_dt")
    return out.value
