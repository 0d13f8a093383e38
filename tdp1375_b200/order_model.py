"""Learned move ordering: data generation, training and installation of the BF16 MLP.

The model scores the C(32,3) = 4960 position triples (i<j<k) of a configuration with
n <= 32 symbols: 1088 inputs (32x32 adjacency of spi in pi-position coordinates + a 64-bin
cycle-length histogram), three hidden layers of 256 (ReLU), 4960 outputs.  All matrix
products run in the library's tcgen05 GEMM (``tdp_mlp_gemm``); torch only holds device
memory.  Training pairs are (state, next move) along the solutions the plain search finds;
the loss is softmax cross-entropy over the triples valid for the state's n.

Installing the model on a slot makes the batched search expand every instance's root
children in descending score order.  Ordering permutes children only, so verdicts do not
change (checked by tests/test_mlp_gpu.py).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from . import native

FEATURES, HIDDEN, TRIPLES, TRIPLES_PADDED = 1088, 256, 4960, 5120
LAYERS = [(HIDDEN, FEATURES), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (TRIPLES_PADDED, HIDDEN)]


def _lex32_table() -> np.ndarray:
    idx = np.full((32, 32, 32), -1, dtype=np.int32)
    t = 0
    for i in range(30):
        for j in range(i + 1, 31):
            for k in range(j + 1, 32):
                idx[i, j, k] = t
                t += 1
    return idx


LEX32 = _lex32_table()


def lib():
    return native.load()


def _check(rc):
    if rc != 0:
        raise RuntimeError(native.last_error() or f"tdp1375 mlp error {rc}")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def gemm(a, b, bias=None, relu=False, out=None, out_fp32=False, stream=None):
    """out[m x n] = a[m x k] @ b[n x k]^T (+bias)(ReLU) on the tensor cores."""
    import torch
    m, k = a.shape
    n = b.shape[0]
    if out is None:
        out = torch.empty(m, n, device=a.device, dtype=torch.float32 if out_fp32 else torch.bfloat16)
    s = ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    _check(lib().tdp_mlp_gemm(_ptr(a), _ptr(b), m, n, k, _ptr(bias) if bias is not None else None, 1 if relu else 0,
                              _ptr(out), 1 if out_fp32 else 0, out.stride(0), s))
    return out


def features(spi, pi, n):
    """spi/pi: uint8 [count x 64] device tensors, n: uint8 [count] -> bf16 [count x 1088]."""
    import torch
    count = spi.shape[0]
    x = torch.empty(count, FEATURES, device=spi.device, dtype=torch.bfloat16)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _check(lib().tdp_mlp_features(_ptr(spi), _ptr(pi), _ptr(n), count, _ptr(x), s))
    return x


@dataclass
class TrainStats:
    steps: int
    pairs: int
    first_loss: float
    last_loss: float
    top1: float


class OrderModel:
    """Weights (bf16 for the GEMMs, fp32 masters for Adam) on the current CUDA device."""

    def __init__(self, seed: int = 1375):
        import torch
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.master, self.weight, self.bias = [], [], []
        for rows, cols in LAYERS:
            w = torch.randn(rows, cols, generator=g) * (2.0 / cols) ** 0.5
            if rows == TRIPLES_PADDED:
                w[TRIPLES:] = 0.0
            self.master.append(w.cuda())
            self.weight.append(w.to(torch.bfloat16).cuda())
            self.bias.append(torch.zeros(rows, device="cuda"))
        self.m = [torch.zeros_like(t) for t in self.master] + [torch.zeros_like(b) for b in self.bias]
        self.v = [torch.zeros_like(t) for t in self.master] + [torch.zeros_like(b) for b in self.bias]
        self.step = 0

    def forward(self, x):
        acts = [x]
        h = x
        for layer in range(3):
            h = gemm(h, self.weight[layer], self.bias[layer], relu=True)
            acts.append(h)
        logits = gemm(h, self.weight[3], self.bias[3], out_fp32=True)
        return logits, acts

    def scores(self, x):
        return self.forward(x)[0]

    def train_step(self, x, n, target, lr=1e-3):
        """One Adam step on a batch; returns (mean loss, top-1 accuracy)."""
        import torch
        L = lib()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rows = x.shape[0]
        logits, acts = self.forward(x)
        dlogits = torch.empty(rows, TRIPLES_PADDED, device=x.device, dtype=torch.bfloat16)
        loss = torch.empty(rows, device=x.device)
        _check(L.tdp_mlp_softmax_xent(_ptr(logits), TRIPLES_PADDED, _ptr(n), _ptr(target), rows, _ptr(dlogits),
                                      _ptr(loss), stream))
        top1 = (logits[:, :TRIPLES].argmax(dim=1) == target.long()).float().mean()
        grads_w, grads_b = [None] * 4, [None] * 4
        grad = dlogits
        for layer in (3, 2, 1, 0):
            a = acts[layer]
            out_dim, in_dim = LAYERS[layer]
            # dW = grad^T @ a : A = grad^T [out x rows], B = a^T [in x rows]
            gT = torch.empty(out_dim, rows, device=x.device, dtype=torch.bfloat16)
            aT = torch.empty(in_dim, rows, device=x.device, dtype=torch.bfloat16)
            _check(L.tdp_mlp_transpose(_ptr(grad), rows, out_dim, _ptr(gT), stream))
            _check(L.tdp_mlp_transpose(_ptr(a), rows, in_dim, _ptr(aT), stream))
            grads_w[layer] = gemm(gT, aT, out_fp32=True)
            gb = torch.empty(out_dim, device=x.device)
            _check(L.tdp_mlp_column_sums(_ptr(grad), rows, out_dim, _ptr(gb), stream))
            grads_b[layer] = gb
            if layer > 0:
                # d(input) = grad @ W : B operand = W^T [in x out]
                wT = torch.empty(in_dim, out_dim, device=x.device, dtype=torch.bfloat16)
                _check(L.tdp_mlp_transpose(_ptr(self.weight[layer]), out_dim, in_dim, _ptr(wT), stream))
                g_in = gemm(grad, wT)
                _check(L.tdp_mlp_relu_backward(_ptr(g_in), _ptr(acts[layer]), g_in.numel(), stream))
                grad = g_in
        self.step += 1
        for layer in range(4):
            _check(L.tdp_mlp_adam(_ptr(self.master[layer]), _ptr(self.weight[layer]), _ptr(grads_w[layer]),
                                  _ptr(self.m[layer]), _ptr(self.v[layer]), self.master[layer].numel(),
                                  ctypes.c_float(lr), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                  ctypes.c_float(1e-8), self.step, stream))
            bias_bf = torch.empty_like(self.bias[layer], dtype=torch.bfloat16)
            _check(L.tdp_mlp_adam(_ptr(self.bias[layer]), _ptr(bias_bf), _ptr(grads_b[layer]), _ptr(self.m[4 + layer]),
                                  _ptr(self.v[4 + layer]), self.bias[layer].numel(), ctypes.c_float(lr),
                                  ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8), self.step, stream))
        with torch.no_grad():
            self.master[3][TRIPLES:] = 0.0
            self.weight[3][TRIPLES:] = 0.0
        return float(loss.mean()), float(top1)

    def install(self, slot: int, enable: bool = True, levels: int = 1) -> None:
        """Copies the weights into the search slot and turns ordering on: levels = 1 orders each
        root's children, 2 also the first level's (enable = False keeps plain order)."""
        import torch
        host_w = [w.contiguous().view(torch.int16).cpu().numpy().astype(np.uint16) for w in self.weight]
        host_w[3] = host_w[3][:TRIPLES]
        host_b = [b.float().cpu().numpy() for b in self.bias]
        host_b[3] = host_b[3][:TRIPLES]
        args = []
        for w, b in zip(host_w, host_b):
            w = np.ascontiguousarray(w)
            b = np.ascontiguousarray(b, dtype=np.float32)
            args += [w.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p)]
            setattr(self, f"_keep_{len(args)}", (w, b))
        _check(lib().tdp_set_order_model(slot, *args))
        _check(lib().tdp_enable_order_model(slot, levels if enable else 0))


def solution_pairs(cases: Sequence[Tuple], results) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(state, next move) pairs along every found solution: spi/pi rows of 64 bytes, n and the
    LEX32 index of the move's positions on the state's pi array."""
    spis, pis, ns, tgts = [], [], [], []
    for case, r in zip(cases, results):
        if r.status != native.FOUND:
            continue
        pi = bytearray(int(v) for v in case[0])
        spi = bytearray(int(v) for v in case[1])
        n = len(pi)
        if n > 32:
            continue
        for d in range(r.depth):
            i, j, k = r.positions[3 * d], r.positions[3 * d + 1], r.positions[3 * d + 2]
            row_s = np.zeros(64, np.uint8)
            row_p = np.zeros(64, np.uint8)
            row_s[:n] = np.frombuffer(bytes(spi), np.uint8)
            row_p[:n] = np.frombuffer(bytes(pi), np.uint8)
            spis.append(row_s)
            pis.append(row_p)
            ns.append(n)
            tgts.append(LEX32[i, j, k])
            a, b, c = pi[i], pi[j], pi[k]
            sa, sb, sc = spi[a], spi[b], spi[c]
            spi[a], spi[b], spi[c] = sc, sa, sb
            pi[i:k] = pi[j:k] + pi[i:j]
    if not spis:
        return (np.zeros((0, 64), np.uint8),) * 2 + (np.zeros(0, np.uint8), np.zeros(0, np.int32))
    return np.stack(spis), np.stack(pis), np.array(ns, np.uint8), np.array(tgts, np.int32)


def train(model: OrderModel, spi: np.ndarray, pi: np.ndarray, n: np.ndarray, target: np.ndarray, epochs: int = 3,
          batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> TrainStats:
    import torch
    rng = np.random.default_rng(seed)
    d_spi, d_pi = torch.from_numpy(spi).cuda(), torch.from_numpy(pi).cuda()
    d_n, d_t = torch.from_numpy(n).cuda(), torch.from_numpy(target).cuda()
    first = last = float("nan")
    acc = 0.0
    steps = 0
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(len(n))).cuda()
        for off in range(0, len(n) - batch + 1, batch):
            idx = perm[off:off + batch]
            x = features(d_spi[idx].contiguous(), d_pi[idx].contiguous(), d_n[idx].contiguous())
            loss, acc = model.train_step(x, d_n[idx].contiguous(), d_t[idx].contiguous(), lr=lr)
            if steps == 0:
                first = loss
            last = loss
            steps += 1
    return TrainStats(steps=steps, pairs=int(len(n)), first_loss=first, last_loss=last, top1=acc)
