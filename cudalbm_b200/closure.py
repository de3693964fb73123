"""Python front end of the learned closure (lbm_trainer_*, lbm_mlp_infer,
lbm_closure_* of include/lbm_b200.h).

Training data come from a fine run filtered 2:1 onto the coarse grid: for a
coarse state F(t) (``coarse.filter_from(fine)``) and the fine run two fine
steps later, ``Trainer.add(coarse, fine)`` stores one sample per selected
interior node (16 features, target dtau) and advances ``coarse`` one step.
``Trainer.fit`` trains the 16 -> 32 -> 32 -> 1 network on the GPU;
``Cavity.set_closure(net)`` makes every later step use it.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional

import numpy as np

from . import _lib


def new_mlp() -> _lib.MLP:
    return _lib.MLP()


class Trainer:
    def __init__(self, capacity: int, device: int = 0):
        t = ctypes.c_void_p()
        _lib.check(_lib.lib().lbm_trainer_create(int(device), int(capacity), ctypes.byref(t)))
        self._t = t

    def close(self) -> None:
        if getattr(self, "_t", None):
            _lib.lib().lbm_trainer_destroy(self._t)
            self._t = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, coarse, fine_next, stride: int = 1, min_neq: float = 0.0) -> int:
        total = ctypes.c_uint64()
        _lib.check(_lib.lib().lbm_trainer_add(self._t, coarse._h, fine_next._h, int(stride), float(min_neq),
                                              ctypes.byref(total)))
        return total.value

    def add_window(self, coarse, fine, window: int, stride: int = 1, min_neq: float = 0.0) -> int:
        """Samples fitted to `window` coarse steps: `coarse` holds the filtered
        state of `fine`, which this advances by 2 x window steps."""
        total = ctypes.c_uint64()
        _lib.check(_lib.lib().lbm_trainer_add_window(self._t, coarse._h, fine._h, int(window), int(stride),
                                                     float(min_neq), ctypes.byref(total)))
        return total.value

    def __len__(self) -> int:
        total = ctypes.c_uint64()
        _lib.check(_lib.lib().lbm_trainer_samples(self._t, 0, 0, None, None, ctypes.byref(total)))
        return total.value

    def samples(self, first: int = 0, count: Optional[int] = None):
        n = len(self) - first if count is None else count
        feats = np.empty((n, 16), np.float32)
        targ = np.empty(n, np.float32)
        _lib.check(_lib.lib().lbm_trainer_samples(self._t, int(first), int(n), feats.ctypes.data, targ.ctypes.data,
                                                  None))
        return feats, targ

    def fit(self, steps: int = 2000, batch: int = 8192, lr: float = 2e-3, dtau_lo: float = -0.002,
            dtau_hi: float = 0.05, seed: int = 0):
        opt = _lib.TrainOptions(steps=int(steps), batch=int(batch), lr=float(lr), dtau_lo=float(dtau_lo),
                                dtau_hi=float(dtau_hi), seed=int(seed))
        net, rep = _lib.MLP(), _lib.TrainReport()
        _lib.check(_lib.lib().lbm_trainer_fit(self._t, ctypes.byref(opt), ctypes.byref(net), ctypes.byref(rep)))
        return net, {f: getattr(rep, f) for f, _ in rep._fields_}

    def gradient(self, net: _lib.MLP, first: int, count: int):
        g, loss = _lib.MLP(), ctypes.c_double()
        _lib.check(_lib.lib().lbm_trainer_gradient(self._t, ctypes.byref(net), int(first), int(count), ctypes.byref(g),
                                                   ctypes.byref(loss)))
        return g, loss.value


def mlp_infer(net: _lib.MLP, features: np.ndarray, tensor_cores: bool = True, device: int = 0) -> np.ndarray:
    """Raw network output for host features [n][16]."""
    f = np.ascontiguousarray(features, dtype=np.float32)
    y = np.empty(f.shape[0], np.float32)
    _lib.check(_lib.lib().lbm_mlp_infer(int(device), ctypes.byref(net), f.ctypes.data, f.shape[0], y.ctypes.data,
                                        int(bool(tensor_cores))))
    return y


def save_mlp(path: str, net: _lib.MLP) -> None:
    np.savez(path, **{name: np.array(getattr(net, name), dtype=np.float32) for name, _ in net._fields_})


def load_mlp(path: str) -> _lib.MLP:
    z = np.load(path)
    net = _lib.MLP()
    for name, ctype in net._fields_:
        v = z[name]
        if v.ndim == 0:
            setattr(net, name, float(v))
        else:
            getattr(net, name)[:] = [float(x) for x in v]
    return net
