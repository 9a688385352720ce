"""Learned SCFT warm start: the spectral neural operator of the library (cfft_sno_*,
include/cfft_b200.h).  No reference counterpart: CrystallographicFFT.jl has no learned
component and no SCFT driver.

A SpectralNeuralOperator holds the weights (FP32 master copy and Adam state on the
device, BF16 working copies); `bind` attaches it to one FP32 KRFFT plan (a group and a
grid) and returns a context that predicts fields [w_A | w_B] for (chiN, f) pairs and
trains on converged fields.  Several contexts of one model share its weights, so one
model learns Im-3m, Ia-3d and Pm-3m together, and a model trained at 64^3 predicts on
any grid of those groups (the input features and spectral weights are functions of
position and Miller index, not of the grid).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import LIB, CFFTError, check
from .plans import _torch

GROUP_SLOTS = {229: 0, 230: 1, 221: 2}  # one-hot order: Im-3m, Ia-3d, Pm-3m


class _Cfg(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_double), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
                ("eps", ctypes.c_double), ("weight_decay", ctypes.c_double)]


_SIGS = {
    "cfft_sno_param_count": (ctypes.c_int64, []),
    "cfft_sno_create": (ctypes.c_int, [ctypes.POINTER(_Cfg), ctypes.POINTER(ctypes.c_void_p)]),
    "cfft_sno_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cfft_sno_set_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cfft_sno_get_params": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cfft_sno_get_grads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cfft_sno_grads_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cfft_sno_apply_grads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "cfft_sno_bind": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "cfft_sno_unbind": (ctypes.c_int, [ctypes.c_void_p]),
    "cfft_sno_predict": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "cfft_sno_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_void_p]),
}
for _n, (_r, _a) in _SIGS.items():
    getattr(LIB, _n).restype = _r
    getattr(LIB, _n).argtypes = _a

N_PARAMS = int(LIB.cfft_sno_param_count())


def _params_array(params):
    a = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1, 2))
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class SpectralNeuralOperator:
    """The network's weights and optimiser state (cfft_sno_create)."""

    def __init__(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        cfg = _Cfg(lr, beta1, beta2, eps, weight_decay)
        h = ctypes.c_void_p()
        check(LIB.cfft_sno_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.lr = lr

    @property
    def handle(self):
        return self._h

    def get_params(self):
        out = np.empty(N_PARAMS, dtype=np.float32)
        check(LIB.cfft_sno_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, values):
        v = np.ascontiguousarray(np.asarray(values, dtype=np.float32).ravel())
        if v.size != N_PARAMS:
            raise CFFTError(1, f"expected {N_PARAMS} parameters, got {v.size}")
        check(LIB.cfft_sno_set_params(self._h, v.ctypes.data))

    def grads(self):
        out = np.empty(N_PARAMS, dtype=np.float32)
        check(LIB.cfft_sno_get_grads(self._h, out.ctypes.data))
        return out

    def grads_device(self, out=None):
        """Gradients of the last train_step as a float32 CUDA tensor (N_PARAMS), copied on
        the current stream: the buffer a data-parallel step averages over ranks."""
        torch = _torch()
        if out is None:
            out = torch.empty(N_PARAMS, dtype=torch.float32, device="cuda")
        elif out.numel() != N_PARAMS or out.dtype != torch.float32 or not (out.is_cuda and out.is_contiguous()):
            raise CFFTError(1, f"out must be a contiguous float32 CUDA tensor of {N_PARAMS} entries")
        check(LIB.cfft_sno_grads_device(self._h, ctypes.c_void_p(out.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return out

    def apply_grads(self, grads=None, lr=None):
        """One Adam step from `grads` (float32 CUDA tensor of N_PARAMS) or, with None, from
        the gradients of the last train_step."""
        torch = _torch()
        ptr = None
        if grads is not None:
            if grads.numel() != N_PARAMS or grads.dtype != torch.float32 or not (grads.is_cuda and grads.is_contiguous()):
                raise CFFTError(1, f"grads must be a contiguous float32 CUDA tensor of {N_PARAMS} entries")
            ptr = ctypes.c_void_p(grads.data_ptr())
        check(LIB.cfft_sno_apply_grads(self._h, ptr, float(self.lr if lr is None else lr),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    def save(self, path):
        """Weights as BF16 bits (the precision the network computes with) in an .npy file."""
        w = self.get_params().view(np.uint32)
        bits = ((w + 0x7FFF + ((w >> 16) & 1)) >> 16).astype(np.uint16)
        np.save(path, bits)

    def load(self, path):
        bits = np.load(path).astype(np.uint32) << 16
        self.set_params(bits.view(np.float32))

    def bind(self, plan, sg, shift, max_samples):
        """Context on `plan` (FP32, group sg in GROUP_SLOTS, shifted by `shift`)."""
        if sg not in GROUP_SLOTS:
            raise CFFTError(4, f"the warm-start network knows groups {sorted(GROUP_SLOTS)}, not {sg}")
        return SNOContext(self, plan, GROUP_SLOTS[sg], shift, max_samples)

    def close(self):
        if getattr(self, "_h", None):
            LIB.cfft_sno_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SNOContext:
    """A model bound to one plan (cfft_sno_bind)."""

    def __init__(self, model, plan, slot, shift, max_samples):
        self.model, self.plan, self.max_samples = model, plan, int(max_samples)
        sh = (ctypes.c_double * 3)(*[float(x) for x in shift])
        h = ctypes.c_void_p()
        check(LIB.cfft_sno_bind(model.handle, plan.handle, int(slot), sh, self.max_samples, ctypes.byref(h)))
        self._h = h

    def _stream(self):
        return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)

    def predict(self, params, out=None):
        """Fields [w_A | w_B] (S, 2, M3, M2, M1) for S pairs (chiN, f)."""
        torch = _torch()
        a, ap = _params_array(params)
        S = a.shape[0]
        shape = (S, 2) + tuple(reversed(self.plan.M))
        if out is None:
            out = torch.empty(shape, dtype=torch.float32, device="cuda")
        elif tuple(out.shape) != shape or out.dtype != torch.float32 or not out.is_contiguous():
            raise CFFTError(1, f"out must be a contiguous float32 tensor of shape {shape}")
        check(LIB.cfft_sno_predict(self._h, ap, S, ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def train_step(self, params, w_target, lr=None, step=True):
        """Loss of the fields w_target (S, 2, M3, M2, M1) and, with step, one Adam update."""
        torch = _torch()
        a, ap = _params_array(params)
        S = a.shape[0]
        if not (w_target.is_cuda and w_target.dtype == torch.float32 and w_target.is_contiguous()
                and w_target.numel() == S * 2 * int(np.prod(self.plan.M))):
            raise CFFTError(1, "w_target must be a contiguous float32 CUDA tensor of S x 2 x M-grid")
        loss = ctypes.c_double()
        check(LIB.cfft_sno_train(self._h, ap, S, ctypes.c_void_p(w_target.data_ptr()),
                                 float(self.model.lr if lr is None else lr), 1 if step else 0, ctypes.byref(loss),
                                 self._stream()))
        return loss.value

    def train_step_data_parallel(self, params, w_target, n_total, dist, lr=None, grad_buf=None):
        """One data-parallel training step over the ranks of a process group (one GPU
        per rank): this rank's samples (params, w_target; possibly none) out of n_total
        in the global mini-batch.  The local gradient of the mean loss is weighted by the
        rank's share of the samples, summed over the ranks by one all-reduce, and every
        rank applies the same Adam step.  Returns the global mean loss."""
        torch = _torch()
        a = np.asarray(params, dtype=np.float64).reshape(-1, 2)
        n_local = a.shape[0]
        g = grad_buf if grad_buf is not None else torch.empty(N_PARAMS + 1, dtype=torch.float32, device="cuda")
        if n_local:
            loss = self.train_step(a, w_target, lr=lr, step=False)
            self.model.grads_device(g[:N_PARAMS])
        else:
            loss = 0.0
            g[:N_PARAMS].zero_()
        total_loss = allreduce_mean_grads(g, loss, n_local, n_total, dist)
        self.model.apply_grads(g[:N_PARAMS], lr=lr)
        return total_loss

    def close(self):
        if getattr(self, "_h", None):
            LIB.cfft_sno_unbind(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_of(indices, rank, world):
    """This rank's slice of a global mini-batch (every world-th sample from `rank`)."""
    return indices[rank::world]


def sample_share(n_local, n_total):
    """Weight of a rank's mean-loss gradient in the global mean: its share of the samples."""
    return float(n_local) / float(n_total) if n_total else 0.0


def allreduce_mean_grads(buf, loss, n_local, n_total, dist):
    """buf = [gradient of this rank's mean loss | one spare entry].  Weights the gradient
    by the rank's share of the samples, puts the weighted loss in the spare entry and
    sums the buffer over the ranks with one all-reduce, so buf[:-1] becomes the gradient
    of the global mean loss on every rank.  Returns the global mean loss."""
    w = sample_share(n_local, n_total)
    buf[:-1].mul_(w)
    buf[-1] = loss * w
    dist.all_reduce(buf)
    return float(buf[-1].item())
