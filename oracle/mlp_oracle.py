"""FP64 NumPy oracle of the warm-start MLP (test infrastructure only).

Layers y = act(x W^T + b), tanh on hidden layers, identity on the last, loss
mean((y - t)^2). The GEMM operands are the layer inputs, the weights, the
backpropagated dZ, the transposed layer inputs and W^T; arith says how a GEMM
treats them, everything else staying FP64:
  "fp64"   plain FP64 products;
  "bf16"   every operand rounded to bfloat16 (round to nearest even on its
           float32 value);
  "split"  the GPU kernels' arithmetic: every operand v (a float32 value) as
           hi = bf16(v) and lo = bf16(v - hi), the product accumulated as
           hi*hi + hi*lo + lo*hi (the lo*lo term dropped).
"""
import numpy as np


def to_bf16(a):
    """Round float values to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, widths):
    Ws, bs, k = [], [], 0
    for l in range(len(widths) - 1):
        i, o = widths[l], widths[l + 1]
        Ws.append(np.asarray(params[k:k + o * i], dtype=np.float64).reshape(o, i))
        k += o * i
        bs.append(np.asarray(params[k:k + o], dtype=np.float64))
        k += o
    return Ws, bs


def pack(Ws, bs):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in zip(Ws, bs)])


def split_bf16(a):
    """hi = bf16(v), lo = bf16(v - hi) of the float32 values v of a (v - hi is exact in float32)."""
    f = np.ascontiguousarray(a, dtype=np.float32).astype(np.float64)
    hi = to_bf16(f)
    return hi, to_bf16(f - hi)


def matmul(a, b, arith="fp64"):
    """a @ b with the operands treated as arith says."""
    if arith == "fp64":
        return np.asarray(a, dtype=np.float64) @ np.asarray(b, dtype=np.float64)
    if arith == "bf16":
        return to_bf16(a) @ to_bf16(b)
    if arith == "split":
        ah, al = split_bf16(a)
        bh, bl = split_bf16(b)
        return al @ bh + ah @ bl + ah @ bh
    raise ValueError(arith)


def forward(params, widths, x, arith="fp64"):
    Ws, bs = unpack(params, widths)
    ys = [np.asarray(x, dtype=np.float64)]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = matmul(ys[-1], W.T, arith) + b
        ys.append(z if l == len(Ws) - 1 else np.tanh(z))
    return ys


def loss_and_grads(params, widths, x, t, arith="fp64"):
    Ws, bs = unpack(params, widths)
    ys = forward(params, widths, x, arith)
    B, O = ys[-1].shape
    d = ys[-1] - np.asarray(t, dtype=np.float64)
    loss = float((d * d).mean())
    dy = 2.0 * d / (B * O)
    gW, gb = [None] * len(Ws), [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        dz = dy if l == len(Ws) - 1 else dy * (1.0 - ys[l + 1] ** 2)
        gb[l] = dz.sum(axis=0)
        gW[l] = matmul(dz.T, ys[l], arith)
        if l > 0:
            dy = matmul(dz, Ws[l], arith)
    return loss, pack(gW, gb)
