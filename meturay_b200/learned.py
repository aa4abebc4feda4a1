"""Learned guiding network (``mrb_mlp_*``): an MLP from a path vertex to a
mixture of 8 von Mises-Fisher lobes over incident directions, trained with
Adam on the tcgen05 tensor cores (BF16 operands, FP32 accumulation)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .tracer import TracerSystem

__all__ = ["GuideMLP", "PARAM_COUNT", "N_IN", "N_OUT"]

PARAM_COUNT = int(lib.mrb_mlp_param_count())
N_IN, N_OUT = 80, 40


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


class GuideMLP:
    def __init__(self, system: TracerSystem, params: np.ndarray | None = None):
        h = C.c_void_p()
        check(lib.mrb_mlp_create(system._h, C.byref(h)))
        self._h = h
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params: np.ndarray):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == PARAM_COUNT
        check(lib.mrb_mlp_set_params(self._h, p.ctypes.data))

    def params(self) -> np.ndarray:
        p = np.zeros(PARAM_COUNT, np.float32)
        check(lib.mrb_mlp_get_params(self._h, p.ctypes.data))
        return p

    @staticmethod
    def encode(pos, nrm, wo, out, stream=None):
        """Device tensors (n x 3 each) -> out (n x 80)."""
        check(lib.mrb_mlp_encode(_ptr(pos), _ptr(nrm), _ptr(wo), int(pos.shape[0]), _ptr(out),
                                 stream))

    def forward(self, features, out, stream=None):
        check(lib.mrb_mlp_forward(self._h, _ptr(features), int(features.shape[0]), _ptr(out),
                                  stream))

    def gradients(self, features, targets, grad, loss, stream=None):
        check(lib.mrb_mlp_gradients(self._h, _ptr(features), _ptr(targets),
                                    int(features.shape[0]), _ptr(grad), _ptr(loss), stream))

    def train_step(self, features, targets, lr: float = 1e-2, stream=None) -> tuple[float, float]:
        out = np.zeros(2, np.float32)
        check(lib.mrb_mlp_train_step(self._h, _ptr(features), _ptr(targets),
                                     int(features.shape[0]), float(lr), out.ctypes.data, stream))
        return float(out[0]), float(out[1])
