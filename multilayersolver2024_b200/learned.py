"""The learned warm start's perceptron (``mlx_mlp_*``): BF16 weights and
activations with FP32 accumulation on the B200 tensor cores, trained with
Adam by the library's own forward and backward kernels."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, f32, load


class Mlp:
    def __init__(self, n_in, n_out, n_hidden=128, n_hidden_layers=3, max_batch=4096, seed=0, device=0):
        lib = load()
        self._lib = lib
        self.n_in, self.n_out = int(n_in), int(n_out)
        h = C.c_void_p()
        check("mlx_mlp_create", lib.mlx_mlp_create(self.n_in, int(n_hidden), int(n_hidden_layers), self.n_out,
                                                    int(max_batch), int(seed), int(device), C.byref(h)), lib)
        self.handle = h
        self.n_hidden, self.n_hidden_layers, self.max_batch = int(n_hidden), int(n_hidden_layers), int(max_batch)

    @property
    def num_params(self) -> int:
        return int(self._lib.mlx_mlp_num_params(self.handle))

    def layer_shapes(self):
        dims = [self.n_in] + [self.n_hidden] * self.n_hidden_layers + [self.n_out]
        return [(dims[i + 1], dims[i]) for i in range(len(dims) - 1)]

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params, np.float32)
        check("mlx_mlp_get_params", self._lib.mlx_mlp_get_params(self.handle, f32(p), p.size), self._lib)
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        check("mlx_mlp_set_params", self._lib.mlx_mlp_set_params(self.handle, f32(p), p.size), self._lib)

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((x.shape[0], self.n_out), np.float32)
        check("mlx_mlp_forward", self._lib.mlx_mlp_forward(self.handle, f32(x), x.shape[0], f32(y)), self._lib)
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_float(0)
        check("mlx_mlp_loss_grad", self._lib.mlx_mlp_loss_grad(self.handle, f32(x), f32(t), x.shape[0], C.byref(loss),
                                                                f32(g)), self._lib)
        return float(loss.value), g

    def train(self, x, t, batch=512, epochs=10, lr=1e-3, seed=0):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        losses = np.zeros(epochs, np.float32)
        check("mlx_mlp_train", self._lib.mlx_mlp_train(self.handle, f32(x), f32(t), x.shape[0], int(batch), int(epochs),
                                                        float(lr), int(seed), f32(losses)), self._lib)
        return losses

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self._lib.mlx_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def collect_warm_start_data(sim, steps, graph=True):
    """Runs `steps` resident steps with recording on (plain solve, mode 0) and
    returns the stacked features (rows x 44), targets (rows x 8) and the
    projectGS iterations of every step (when the step monitors residuals)."""
    sim.warm_start(record=True, mode=0)
    feats, tgts, iters = [], [], []
    for _ in range(steps):
        sim.step(1, graph=graph)
        f, t = sim.warm_start_records()
        feats.append(f)
        tgts.append(t)
        try:
            iters.append(sim.monitor()[1])
        except Exception:
            iters.append(None)
    return np.concatenate(feats), np.concatenate(tgts), iters


def normalisation(a, floor=1e-6):
    a = np.asarray(a, np.float64)
    return a.mean(0).astype(np.float32), np.maximum(a.std(0), floor).astype(np.float32)


def fit_warm_start(features, targets, epochs=200, lr=2e-3, batch=None, seed=0, hidden=128, layers=3, max_batch=4096):
    """Trains the warm-start perceptron (44 -> 8) on normalised features and
    targets with the library's tensor-core kernels.  Returns the network, the
    feature and output normalisations and the per-epoch losses."""
    fn, on = normalisation(features), normalisation(targets)
    x = (features - fn[0]) / fn[1]
    y = (targets - on[0]) / on[1]
    n = x.shape[0]
    b = batch or min(max(128, n // 8 // 128 * 128), max_batch)
    b = min(b, n)
    net = Mlp(44, 8, n_hidden=hidden, n_hidden_layers=layers, max_batch=max(max_batch, b), seed=seed)
    losses = net.train(x, y, batch=b, epochs=epochs, lr=lr, seed=seed)
    return net, fn, on, losses


def predict(net, fn, on, features):
    """Denormalised outputs of the warm-start network."""
    return net.forward((features - fn[0]) / fn[1]) * on[1] + on[0]
