"""Oracle of the learned-preconditioner network (test infrastructure only).

Float64 numpy forward and backward of the per-plane-wave MLP of
``gradwave_b200/csrc/mlp.cu`` (4 -> 64 -> 64 -> 64 -> 1, SiLU), emulating its
BF16 rounding of weights, inputs and hidden activations (round to nearest
even), with the loss sum_i w_i (o_i - y_i)^2 and straight-through gradients
for the rounded weights. The reference has no learned preconditioner; this
oracle checks the CUDA training kernels, whose gradients must match it to
float32 accumulation error.
"""

from __future__ import annotations

import numpy as np

HID, NIN = 64, 4
SHAPES = [("W1", (HID, NIN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (HID,)), ("b4", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SHAPES])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float64 values to bfloat16 (via float32, nearest even)."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p: np.ndarray, u: np.ndarray, emulate_bf16: bool = True):
    q = unpack(p)
    rnd = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    W = {k: (rnd(v) if k != "b4" else rnd(v)) for k, v in q.items()}
    a0 = rnd(u)
    z1 = a0 @ W["W1"].T + W["b1"]
    a1 = rnd(z1 * _sig(z1))
    z2 = a1 @ W["W2"].T + W["b2"]
    a2 = rnd(z2 * _sig(z2))
    z3 = a2 @ W["W3"].T + W["b3"]
    a3 = rnd(z3 * _sig(z3))
    o = a3 @ W["W4"] + W["b4"][0]
    return o, (W, a0, z1, a1, z2, a2, z3, a3)


def loss_grad(p, u, y, w, emulate_bf16: bool = True):
    """(loss, gradient) of sum_i w_i (o_i - y_i)^2."""
    o, (W, a0, z1, a1, z2, a2, z3, a3) = forward(p, u, emulate_bf16)
    e = o - y
    loss = float(np.sum(w * e * e))
    do = 2.0 * w * e

    def dsilu(z):
        s = _sig(z)
        return s * (1.0 + z * (1.0 - s))

    g = {"W4": a3.T @ do, "b4": np.array([do.sum()])}
    dz3 = do[:, None] * W["W4"][None, :] * dsilu(z3)
    g["W3"] = dz3.T @ a2
    g["b3"] = dz3.sum(0)
    dz2 = (dz3 @ W["W3"]) * dsilu(z2)
    g["W2"] = dz2.T @ a1
    g["b2"] = dz2.sum(0)
    dz1 = (dz2 @ W["W2"]) * dsilu(z1)
    g["W1"] = dz1.T @ a0
    g["b1"] = dz1.sum(0)
    return loss, pack(g)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation with a zero output layer (the network starts as
    the identity correction, K = TPA)."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.standard_normal((HID, NIN)) * np.sqrt(2.0 / NIN), "b1": np.zeros(HID),
         "W2": rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID), "b2": np.zeros(HID),
         "W3": rng.standard_normal((HID, HID)) * np.sqrt(2.0 / HID), "b3": np.zeros(HID),
         "W4": np.zeros(HID), "b4": np.zeros(1)}
    return pack(d)
