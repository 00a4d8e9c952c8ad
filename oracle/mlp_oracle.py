"""TEST INFRASTRUCTURE ONLY -- FP64 numpy restatement of the warm-start MLP (no reference
counterpart): forward pass, mean-squared-error loss and its analytic gradient, with the parameter
layout of libsovipm's sov_mlp (per layer W (out x in, row-major) then b). The GPU kernels run the
same network with BF16 operands and FP32 accumulation; tests compare their loss and gradients
with this restatement at BF16 tolerance."""
from __future__ import annotations

import numpy as np


def unpack(params: np.ndarray, dims: list[int]):
    ws, bs, off = [], [], 0
    for l in range(len(dims) - 1):
        n_out, n_in = dims[l + 1], dims[l]
        ws.append(params[off:off + n_out * n_in].reshape(n_out, n_in).astype(np.float64))
        off += n_out * n_in
        bs.append(params[off:off + n_out].astype(np.float64))
        off += n_out
    return ws, bs


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to BF16 (round to nearest, ties to even) and back, as the kernels stage operands."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    u = ((u + (np.uint32(0x7FFF) + ((u >> np.uint32(16)) & np.uint32(1)))) & np.uint32(0xFFFF0000)).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def loss_and_grad(params: np.ndarray, dims: list[int], x: np.ndarray, t: np.ndarray, bf16_operands: bool = False):
    """Exact FP64 (default) or with every product operand rounded to BF16 first (the kernels'
    arithmetic: BF16 operands, wide accumulation, FP32 storage of results)."""
    r = bf16 if bf16_operands else (lambda a: np.asarray(a, dtype=np.float64))
    f = (lambda a: a.astype(np.float32).astype(np.float64)) if bf16_operands else (lambda a: a)
    ws, bs = unpack(params, dims)
    acts = [f(x.astype(np.float64))]
    for l, (w, b) in enumerate(zip(ws, bs)):
        z = f(r(acts[-1]) @ r(w).T + b)
        acts.append(np.maximum(z, 0.0) if l + 1 < len(ws) else z)
    diff = acts[-1] - t
    loss = float(np.mean(diff ** 2))
    d = f(2.0 * diff / diff.size)
    grads = [None] * (2 * len(ws))
    for l in range(len(ws) - 1, -1, -1):
        grads[2 * l] = r(d).T @ r(acts[l])
        grads[2 * l + 1] = d.sum(axis=0)
        if l > 0:
            d = f(r(d) @ r(ws[l])) * (acts[l] > 0)
    flat = np.concatenate([g.reshape(-1) for g in grads])
    return loss, flat, acts[-1]
