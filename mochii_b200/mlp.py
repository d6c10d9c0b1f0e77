"""Learned warm start of the thermal balance (C-ABI wrapper).

A 4-layer MLP (16 -> 128 -> 128 -> 128 -> 4, GELU), trained on the GPU by
the library's own BF16 tensor-core kernels on (leaf features, solved leaf
state) pairs that the cell solver produces.  Its T_e prediction seeds the
bracketed thermal solve (par thermal_solver = 'bracketed'), which solves
every leaf to the usual tolerance from there; a poor prediction costs
solver evaluations, never accuracy.

    mlp = WarmStartMLP(seed=1)
    X, Y = [], []
    for it in range(niter):                       # plain iterations make data
        neb.ionizing_field_and_rates()
        X.append(WarmStartMLP.features(neb))
        neb.gas_thermal_update()
        Y.append(WarmStartMLP.targets(neb, X[-1]))
    mlp.train(np.concatenate(X), np.concatenate(Y), epochs=20)
    neb.ionizing_field_and_rates()
    mlp.warm_start(neb)                            # predicted T_e -> the solver
    neb.gas_thermal_update()
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import MochiiError

NIN, NOUT, HID, LAYERS = 16, 4, 128, 4
DIMS = [NIN, HID, HID, HID, NOUT]


class WarmStartMLP:
    def __init__(self, seed=0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.mochii_mlp_create(int(seed), C.byref(h))
        if rc:
            raise MochiiError(rc, "mochii_mlp_create failed")
        self.h = h

    def _ok(self, rc):
        if rc:
            msg = self.lib.mochii_mlp_last_error(self.h)
            raise MochiiError(rc, msg.decode() if msg else "")

    def close(self):
        if self.h:
            self.lib.mochii_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def num_params():
        return int(_lib.load().mochii_mlp_num_params())

    def params(self):
        p = np.zeros(self.num_params(), dtype=np.float32)
        self._ok(self.lib.mochii_mlp_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params()
        self._ok(self.lib.mochii_mlp_set_params(self.h, p.ctypes.data))

    def gradients(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(self.num_params(), dtype=np.float32)
        loss = C.c_float()
        self._ok(self.lib.mochii_mlp_gradients(self.h, X.ctypes.data, Y.ctypes.data, X.shape[0], g.ctypes.data,
                                               C.byref(loss)))
        return g, loss.value

    def train(self, X, Y, epochs=10, batch=4096, lr=1e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        self._ok(self.lib.mochii_mlp_train(self.h, X.ctypes.data, Y.ctypes.data, X.shape[0], int(epochs), int(batch),
                                           float(lr), int(seed), losses.ctypes.data))
        return losses

    def predict(self, X):
        """(n, 4): x_HII, x_HeII, x_HeIII, T_e [K]."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros((X.shape[0], 4))
        self._ok(self.lib.mochii_mlp_predict(self.h, X.ctypes.data, X.shape[0], out.ctypes.data))
        return out

    def warm_start(self, neb):
        """The predicted T_e of every leaf seeds the next bracketed thermal solve."""
        self._ok(self.lib.mochii_mlp_warm_start(neb.ctx, self.h))

    @staticmethod
    def features(neb):
        X = np.zeros((neb.nleaf, NIN), dtype=np.float32)
        rc = neb.lib.mochii_mlp_features(neb.ctx, X.ctypes.data)
        if rc:
            raise MochiiError(rc, "mochii_mlp_features failed")
        return X

    @staticmethod
    def targets(neb, X):
        """The solved state as training targets for the features X taken
        before the solve: x_HII, x_HeII, x_HeIII and 4 (log10 T_e - log10
        T_e,prev), the previous T_e being the one feature 11 encodes."""
        xHI, h1, h2, T = neb.get("x_HI"), neb.get("x_HeI"), neb.get("x_HeII"), neb.get("T_e")
        lprev = 4.0 + X[:, 11].astype(np.float64) / 4.0
        return np.stack([1.0 - xHI, h2, np.maximum(0.0, 1.0 - h1 - h2), 4.0 * (np.log10(T) - lprev)],
                        axis=1).astype(np.float32)
