"""Learned warm starts for a parametric LP family.

An MLP (hand-written BF16 tensor-core kernels in libsovipm, FP32 master weights, Adam) maps the
family's instance parameters (the multiplicative perturbations of b and c) to an interior iterate
(x, y, s) of the engine's own standard form: the point the IPM reaches after k steps from its
default start, on the early, well-centred stretch of the central path (a final, nearly
complementary solution is a poor interior start: pushed back into the interior it costs more
iterations than it saves). It is trained on iterates the IPM itself produces. At solve time the
prediction is floored (x, s >= delta) and handed to the engine, which rejects gross mispredictions
(residual metric 10x worse than the default start's); every run is driven to the same FP64
tolerances, so the warm start changes the iteration count, never the answer's accuracy.

No counterpart in the reference (the reference starts every solve from
solver/lp/src/interior_point.cpp:488-506).
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from ._lib import check, load
from .ipm import InteriorPointOptions, InteriorPointSolver
from .model import Model, Result


class Mlp:
    """sov_mlp: n_in -> hidden x layers (ReLU) -> n_out."""

    def __init__(self, n_in: int, n_out: int, hidden: int = 512, layers: int = 3, seed: int = 0):
        self.dims = [n_in] + [hidden] * layers + [n_out]
        h = C.c_void_p()
        check(load().sov_mlp_create(n_in, hidden, layers, n_out, seed, C.byref(h)))
        self.h = h
        self.nparam = int(load().sov_mlp_param_count(h))

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.nparam, dtype=np.float32)
        check(load().sov_mlp_get_params(self.h, p.ctypes.data, self.nparam))
        return p

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(load().sov_mlp_set_params(self.h, p.ctypes.data, self.nparam))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.dims[-1]), dtype=np.float32)
        check(load().sov_mlp_forward(self.h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def loss_grad(self, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = C.c_double()
        check(load().sov_mlp_loss_grad(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], C.byref(loss), g.ctypes.data))
        return loss.value, g

    def train(self, x: np.ndarray, t: np.ndarray, epochs: int, batch: int = 256, lr: float = 1e-3,
              seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_double()
        check(load().sov_mlp_train(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], epochs, batch, lr, seed,
                                   C.byref(loss)))
        return loss.value

    def close(self) -> None:
        if self.h:
            load().sov_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_many(models: list[Model], options: InteriorPointOptions | None = None, warm: list | None = None,
               workers: int = 8) -> tuple[list[Result], float]:
    """Independent single-problem solves, `workers` at a time on separate CUDA streams."""
    solver = InteriorPointSolver(options or InteriorPointOptions())

    def one(k):
        return solver.solve(models[k], with_ipm=True, with_diag=True,
                            warm_start=None if warm is None else warm[k])

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        res = list(ex.map(one, range(len(models))))
    return res, time.perf_counter() - t0


@dataclass
class Normalizer:
    mean: np.ndarray
    std: np.ndarray

    @classmethod
    def fit(cls, a: np.ndarray) -> "Normalizer":
        return cls(a.mean(axis=0), np.maximum(a.std(axis=0), 1e-6))

    def apply(self, a):
        return (a - self.mean) / self.std

    def invert(self, a):
        return a * self.std + self.mean


class WarmStart:
    """Parameter vector -> (x, y, s) predictor for one LP family (fixed A, perturbed b and c)."""

    FLOOR = 1e-14

    def __init__(self, n_param: int, n_ipm: int, m_ipm: int, hidden: int = 512, layers: int = 3, seed: int = 0):
        self.n_ipm, self.m_ipm = n_ipm, m_ipm
        self.mlp = Mlp(n_param, 2 * n_ipm + m_ipm, hidden, layers, seed)
        self.fin: Normalizer | None = None
        self.fout: Normalizer | None = None

    def _targets(self, results: list[Result]) -> np.ndarray:
        t = np.stack([np.concatenate([np.log(np.maximum(r.ipm_x, self.FLOOR)), r.ipm_y,
                                      np.log(np.maximum(r.ipm_s, self.FLOOR))]) for r in results])
        return t

    def targets(self, results: list[Result]) -> tuple[np.ndarray, np.ndarray]:
        """(indices of the OPTIMAL results, their training targets): log x, y, log s of the captured
        iterate. Lets a caller generate a large training set in chunks and drop the results."""
        ok = [k for k, r in enumerate(results) if r.status_name == "OPTIMAL"]
        return np.array(ok, dtype=np.int64), self._targets([results[k] for k in ok])

    def fit(self, params: np.ndarray, results: list[Result], epochs: int = 60, batch: int = 128, lr: float = 1e-3,
            seed: int = 0) -> float:
        ok, t = self.targets(results)
        return self.fit_arrays(params[ok], t, epochs, batch, lr, seed)

    def fit_arrays(self, params: np.ndarray, targets: np.ndarray, epochs: int = 60, batch: int = 128,
                   lr: float = 1e-3, seed: int = 0) -> float:
        """Normalizers and network from parameter rows and their targets (see targets())."""
        self.fin, self.fout = Normalizer.fit(params), Normalizer.fit(targets)
        return self.mlp.train(self.fin.apply(params), self.fout.apply(targets), epochs, batch, lr, seed)

    def predict(self, params: np.ndarray, delta: float = 1e-6) -> list[tuple[np.ndarray, np.ndarray, np.ndarray]]:
        """Warm starts floored into the interior: x, s >= delta (scaled problem units). Normalization,
        the network and the decoding (x = max(exp(clip(log x, -40, 40)), delta), likewise s) run on
        the GPU in one call (sov_mlp_predict_start)."""
        p = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        n, m, b = self.n_ipm, self.m_ipm, p.shape[0]
        xs, ys, ss = np.empty((b, n)), np.empty((b, m)), np.empty((b, n))
        f = [np.ascontiguousarray(v, dtype=np.float64) for v in (self.fin.mean, self.fin.std, self.fout.mean,
                                                                  self.fout.std)]
        check(load().sov_mlp_predict_start(self.mlp.h, p.ctypes.data, b, *(v.ctypes.data for v in f), n, m, delta,
                                           xs.ctypes.data, ys.ctypes.data, ss.ctypes.data))
        return [(xs[k], ys[k], ss[k]) for k in range(b)]

    def solve_batch(self, models, params: np.ndarray, delta: float = 1e-6, options=None, with_diag: bool = False):
        """The batch solved from the network's starts without their leaving the device
        (sov_lp_solve_batch_predicted): the same results as solve_batch(models,
        warm_starts=self.predict(params)), minus the starts' round trip through host memory."""
        import ctypes as C
        from . import abi
        from .ipm import InteriorPointOptions
        from .model import ResultBuffers
        p = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        if p.shape[0] != len(models):
            raise ValueError("one parameter row per model")
        f = [np.ascontiguousarray(v, dtype=np.float64) for v in (self.fin.mean, self.fin.std, self.fout.mean,
                                                                  self.fout.std)]
        opt = (options or InteriorPointOptions()).to_abi()
        bufs = [ResultBuffers(m, with_diag=with_diag) for m in models]
        arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
        res = (abi.SovResult * len(models))(*[b.raw for b in bufs])
        check(load().sov_lp_solve_batch_predicted(self.mlp.h, p.ctypes.data, *(v.ctypes.data for v in f), self.n_ipm,
                                                  self.m_ipm, delta, len(models), arr, C.byref(opt), res))
        out = []
        for b, r in zip(bufs, res):
            b.raw = r
            out.append(b.to_result())
        return out
