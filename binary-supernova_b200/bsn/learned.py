"""Learned WENO weights: sample collection, GPU training and installation.

The networks and their fallback rule are described in include/bsn.h (section
"learned WENO weights").  Everything here runs on the GPU through libbsn:
collect_samples() gathers (normalised stencil, FP64 WENO-Z weights) pairs
from a state the method itself produced, train() runs the hand-written
forward/backward/Adam kernels, install() packs the parameters to BF16 for the
tensor-core inference inside the stencil kernel.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from ._lib import BSNError, load
from .api import BC, NG, _call, _check_state, _ptr, context

NPARAM = None
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weno_mlp.npz")


def nparam() -> int:
    global NPARAM
    if NPARAM is None:
        NPARAM = int(load().bsn_learned_param_count())
    return NPARAM


def _fptr(t: torch.Tensor):
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError("expected a contiguous CUDA float32 tensor")
    return C.c_void_p(t.data_ptr())


class SampleBuffers:
    """Device buffers of training samples for the left and right networks."""

    def __init__(self, cap: int, device="cuda"):
        self.cap = int(cap)
        self.L = torch.empty((self.cap, 8), device=device, dtype=torch.float32)
        self.R = torch.empty((self.cap, 8), device=device, dtype=torch.float32)
        self.counts = (C.c_longlong * 2)(0, 0)

    def collect(self, U, nx, ny, nz, gamma, *, stride=1, seed=0, bc="outflow"):
        _check_state(U, nx, ny, nz)
        _call("bsn_learned_collect", context(), _ptr(U), nx, ny, nz, BC[bc], float(gamma), int(stride),
              C.c_ulonglong(seed), _fptr(self.L), _fptr(self.R), C.c_longlong(self.cap), self.counts)
        return tuple(self.counts)

    @property
    def stored(self):
        return min(self.counts[0], self.cap), min(self.counts[1], self.cap)

    def left(self):
        return self.L[: self.stored[0]]

    def right(self):
        return self.R[: self.stored[1]]


IDEAL = {0: (0.1, 0.6, 0.3), 1: (0.3, 0.6, 0.1)}   # linear weights of src/weno5.jl:37,57


def init_params(seed: int = 0, side: int | None = None) -> torch.Tensor:
    """Parameters of one network (FP32, device).  Hidden layers He-initialised.
    With `side` given the output starts at the linear (ideal) weights of that
    side -- bias log(d), last layer near zero -- so the network learns a
    correction to them; the FP32 bias also keeps BF16 rounding of the hidden
    activations confined to that (small) correction."""
    rng = np.random.default_rng(seed)
    p = np.zeros(nparam(), dtype=np.float32)
    o = 0
    for layer, (nout, nin) in enumerate(((32, 5), (32, 32), (3, 32))):
        scale = np.sqrt(2.0 / nin) * (0.01 if (layer == 2 and side is not None) else 1.0)
        p[o:o + nout * nin] = rng.standard_normal(nout * nin) * scale
        o += nout * nin
        p[o:o + nout] = np.log(IDEAL[side]) if (layer == 2 and side is not None) else 0.0
        o += nout
    return torch.from_numpy(p).cuda()


def grad(samples: torch.Tensor, params: torch.Tensor):
    g = torch.zeros(nparam(), device=samples.device, dtype=torch.float32)
    loss = C.c_double()
    _call("bsn_learned_grad", context(), _fptr(samples), C.c_longlong(samples.shape[0]), _fptr(params), _fptr(g),
          C.byref(loss))
    return g, loss.value


def train(samples: torch.Tensor, params: torch.Tensor, *, steps=2000, batch=4096, lr=3e-3, seed=0) -> float:
    loss = C.c_double()
    _call("bsn_learned_train", context(), _fptr(samples), C.c_longlong(samples.shape[0]), _fptr(params),
          int(steps), int(batch), C.c_float(lr), C.c_ulonglong(seed), C.byref(loss))
    return loss.value


def evaluate(u: torch.Tensor, params: torch.Tensor, tensor_cores=True) -> torch.Tensor:
    n = u.shape[0]
    w = torch.empty((n, 3), device=u.device, dtype=torch.float32)
    _call("bsn_learned_eval", context(), _fptr(u.contiguous()), C.c_longlong(n), _fptr(params), _fptr(w),
          int(bool(tensor_cores)))
    return w


def install(params_left: torch.Tensor, params_right: torch.Tensor):
    _call("bsn_learned_set_params", context(), _fptr(params_left), _fptr(params_right))


def save(path, params_left, params_right, **meta):
    np.savez(path, left=params_left.cpu().numpy(), right=params_right.cpu().numpy(),
             **{k: np.asarray(v) for k, v in meta.items()})


def load_params(path=DEFAULT_PATH):
    d = np.load(path)
    return torch.from_numpy(d["left"]).cuda(), torch.from_numpy(d["right"]).cuda()
