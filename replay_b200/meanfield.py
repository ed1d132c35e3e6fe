"""Differentiable expected-value (mean-field) replay as a torch op.

`MeanField(graph, iterations=..., ...)` holds the schedule and every window
CSR of a replay on the graph's GPU (rp_meanfield_create).  Calling it runs
the forward kernels on the current torch stream and returns

    incidence  (iterations,)  expected new infections per step
    x_T        (4, N)         final S, E, I, R probabilities

through the op `torch.ops.replay_b200.meanfield`, registered with the torch
dispatcher (torch.library.custom_op, with a fake implementation for shape
propagation) and with the hand-written reverse-time adjoint
(rp_meanfield_backward) as its autograd formula: gradients flow to x0, beta,
the per-node susceptibility and the E->I, I->R, R->S rates.  The library
replays the whole forward (and adjoint) as one captured CUDA graph.

    mf = MeanField(g, iterations=336, step_size=3600, window=3600, start_time=t0)
    inc, xT = mf(x0, beta, susceptibility=s, p_ei=1/48, p_ir=1/120)
    loss = ((inc.view(-1, 24).sum(1) - target) ** 2).mean()
    loss.backward()

Everything runs on the GPU through libreplay; there is no CPU path.
"""
import ctypes as C
import math
from typing import Optional, Tuple

import torch

from . import _lib
from ._lib import check, lib

__all__ = ["MeanField", "meanfield_op", "daily_incidence", "calibrate_beta"]


def _scalar(v, like):
    if isinstance(v, torch.Tensor):
        return v
    return torch.tensor(float(v), dtype=torch.float32, device=like.device)


# Live MeanField objects by handle id: the registered op takes the id (an
# int) in place of the Python object.
_LIVE = {}


def _f32(t):
    """A contiguous float32 tensor with t's values (t itself when it is one)."""
    if t is None or (t.dtype == torch.float32 and t.is_contiguous()):
        return t
    return t.to(torch.float32).contiguous()


@torch.library.custom_op("replay_b200::meanfield", mutates_args=())
def meanfield_op(handle: int, x0: torch.Tensor, beta: torch.Tensor, sus: Optional[torch.Tensor],
                 p_ei: torch.Tensor, p_ir: torch.Tensor, p_rs: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """Expected-value replay of MeanField `handle` (rp_meanfield_forward):
    returns (incidence (T,), x_T (4, N)) in float32 on the graph's GPU."""
    mf = _LIVE[handle]
    return mf._forward(_f32(x0), _f32(sus), [float(v) for v in (beta, p_ei, p_ir, p_rs)])


@meanfield_op.register_fake
def _(handle, x0, beta, sus, p_ei, p_ir, p_rs):
    mf = _LIVE[handle]
    return x0.new_empty((mf.T,), dtype=torch.float32), x0.new_empty((4, mf.N), dtype=torch.float32)


def _setup_context(ctx, inputs, output):
    handle, x0, beta, sus, p_ei, p_ir, p_rs = inputs
    mf = _LIVE[handle]
    ctx.handle = handle
    ctx.generation = mf._generation
    ctx.inputs = (_f32(x0.detach()), _f32(sus.detach()) if sus is not None else None,
                  [float(v) for v in (beta, p_ei, p_ir, p_rs)])
    ctx.has_sus = sus is not None
    ctx.rate_dtypes = [v.dtype for v in (beta, p_ei, p_ir, p_rs)]


def _backward(ctx, g_inc, g_xT):
    """The reverse-time adjoint (rp_meanfield_backward)."""
    mf = _LIVE[ctx.handle]
    if mf._generation != ctx.generation:  # another forward ran since: restore its checkpoints
        mf._forward(*ctx.inputs)
    dev = mf.device
    g_inc, g_xT = _f32(g_inc), _f32(g_xT)
    gx0 = torch.empty((4, mf.N), dtype=torch.float32, device=dev)
    gsus = torch.empty(mf.N, dtype=torch.float32, device=dev) if ctx.has_sus else None
    grates = torch.empty(4, dtype=torch.float64, device=dev)
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    check(lib().rp_meanfield_backward(mf._h, ptr(g_inc), ptr(g_xT), ptr(gx0), ptr(gsus), ptr(grates),
                                      C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))
    g = [grates[k].to(ctx.rate_dtypes[k]) for k in range(4)]
    return None, gx0, g[0], gsus, g[1], g[2], g[3]


meanfield_op.register_autograd(_backward, setup_context=_setup_context)


class MeanField:
    """Expected-value replay over a Graph's per-step window CSRs.

    Keyword arguments follow Simulation: iterations (n_steps), step_size,
    start_time, window, has_exposed, ir_to_s, ncls_cap; checkpoint_every is
    the adjoint's checkpoint interval in steps (states in between are
    recomputed)."""

    _ALIASES = {"iterations": "n_steps", "static_network_duration": "window"}

    def __init__(self, graph, checkpoint_every=24, **kw):
        p = _lib.Params()
        lib().rp_params_default(C.byref(p))
        for k, val in kw.items():
            k = self._ALIASES.get(k, k)
            if k in ("ncls_cap", "has_exposed", "ir_to_s"):
                val = int(bool(val))
            if k not in ("n_steps", "step_size", "start_time", "window", "ncls_cap", "has_exposed", "ir_to_s"):
                raise TypeError(f"unknown mean-field parameter {k!r}")
            setattr(p, k, val)
        self.graph = graph
        self.N = graph.n_nodes
        self.T = p.n_steps
        self.device = torch.device("cuda", graph.info["device"])
        h = C.c_void_p()
        check(lib().rp_meanfield_create(graph._h, C.byref(p), int(checkpoint_every), C.byref(h)))
        self._h = h
        self._generation = 0
        self.handle = h.value
        _LIVE[self.handle] = self

    def _forward(self, x0, sus, rates):
        if x0.shape != (4, self.N) or x0.device != self.device:
            raise ValueError(f"x0 must be a (4, {self.N}) tensor on {self.device}")
        if sus is not None and (sus.shape != (self.N,) or sus.device != self.device):
            raise ValueError(f"susceptibility must be a ({self.N},) tensor on {self.device}")
        inc = torch.empty(self.T, dtype=torch.float32, device=self.device)
        xT = torch.empty((4, self.N), dtype=torch.float32, device=self.device)
        beta, p_ei, p_ir, p_rs = rates
        check(lib().rp_meanfield_forward(
            self._h, C.c_void_p(x0.data_ptr()), beta, C.c_void_p(sus.data_ptr()) if sus is not None else None,
            p_ei, p_ir, p_rs, C.c_void_p(inc.data_ptr()), C.c_void_p(xT.data_ptr()),
            C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
        self._generation += 1
        return inc, xT

    def __call__(self, x0, beta, susceptibility=None, p_ei=0.0, p_ir=0.0, p_rs=0.0):
        x0 = x0.reshape(4, self.N)
        beta = _scalar(beta, x0)
        p_ei, p_ir, p_rs = (_scalar(v, x0) for v in (p_ei, p_ir, p_rs))
        return torch.ops.replay_b200.meanfield(self.handle, x0, beta, susceptibility, p_ei, p_ir, p_rs)

    def close(self):
        if self._h and self._h.value:
            _LIVE.pop(self.handle, None)
            lib().rp_meanfield_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def daily_incidence(incidence, steps_per_day):
    """Sums per-step incidence into days (trailing partial day dropped)."""
    days = incidence.shape[-1] // steps_per_day
    return incidence[..., :days * steps_per_day].reshape(*incidence.shape[:-1], days, steps_per_day).sum(-1)


def calibrate_beta(mf, x0, target_daily, beta0, steps_per_day=24, susceptibility=None, p_ei=0.0, p_ir=0.0,
                   p_rs=0.0, iters=60, lr=0.1):
    """Fits the global transmission rate beta so that the mean-field daily
    incidence matches `target_daily` in mean squared error (Adam on log beta,
    gradients from the adjoint).  Returns (beta, per-iteration losses)."""
    dev = mf.device
    target = torch.as_tensor(target_daily, dtype=torch.float32, device=dev)
    x0 = torch.as_tensor(x0, dtype=torch.float32, device=dev)
    logb = torch.tensor(math.log(beta0), dtype=torch.float32, device=dev, requires_grad=True)
    opt = torch.optim.Adam([logb], lr=lr)
    losses = []
    for _ in range(iters):
        opt.zero_grad()
        inc, _ = mf(x0, logb.exp(), susceptibility=susceptibility, p_ei=p_ei, p_ir=p_ir, p_rs=p_rs)
        loss = ((daily_incidence(inc, steps_per_day) - target) ** 2).mean()
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    return float(logb.detach().exp()), losses
