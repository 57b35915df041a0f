"""FP64 NumPy oracle of the warm-start MLP (test infrastructure only).

Layers y = act(x W^T + b), tanh on hidden layers, identity on the last, loss
mean((y - t)^2). With bf16=True every GEMM operand is rounded to bfloat16 the
way the GPU kernels round it (round to nearest even on the float32 value):
the layer inputs, the weights, the backpropagated dZ, the transposed layer
inputs and W^T; everything else stays FP64.
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


def forward(params, widths, x, bf16=False):
    Ws, bs = unpack(params, widths)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    ys = [np.asarray(x, dtype=np.float64)]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = r(ys[-1]) @ r(W).T + b
        ys.append(z if l == len(Ws) - 1 else np.tanh(z))
    return ys


def loss_and_grads(params, widths, x, t, bf16=False):
    Ws, bs = unpack(params, widths)
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    ys = forward(params, widths, x, bf16)
    B, O = ys[-1].shape
    d = ys[-1] - np.asarray(t, dtype=np.float64)
    loss = float((d * d).mean())
    dy = 2.0 * d / (B * O)
    gW, gb = [None] * len(Ws), [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        dz = dy if l == len(Ws) - 1 else dy * (1.0 - ys[l + 1] ** 2)
        gb[l] = dz.sum(axis=0)
        gW[l] = r(dz).T @ r(ys[l])
        if l > 0:
            dy = r(dz) @ r(Ws[l])
    return loss, pack(gW, gb)
