"""Test infrastructure only: FP64 NumPy oracle of the learned warm-start
network (20 -> 64 -> 64 -> 64 -> 3, GELU, standardised inputs/outputs) and
of its loss gradient.

BF16 rounding is applied at the same points as the CUDA kernels (weights,
layer inputs, back-propagated pre-activation gradients) so the check isolates
accumulation order (FP32 on the tensor cores vs FP64 here).  The parameter
layout is the flat vector of include/chysx_cloth.h (chysx_cloth_set_network).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

N_IN, N_HID, N_OUT = 20, 64, 3


def offsets():
    o = {}
    k = 0
    for name, size in (("mu_in", N_IN), ("sd_in", N_IN), ("mu_out", N_OUT), ("sd_out", N_OUT),
                       ("w1", N_IN * N_HID), ("b1", N_HID), ("w2", N_HID * N_HID), ("b2", N_HID),
                       ("w3", N_HID * N_HID), ("b3", N_HID), ("w4", N_HID * N_OUT), ("b4", N_OUT)):
        o[name] = (k, k + size)
        k += size
    o["total"] = k
    return o


OFF = offsets()


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    x32 = np.ascontiguousarray(x, np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    g = {k: p[v[0]:v[1]] for k, v in OFF.items() if k != "total"}
    return dict(mu_in=g["mu_in"], sd_in=g["sd_in"], mu_out=g["mu_out"], sd_out=g["sd_out"],
                w1=g["w1"].reshape(N_IN, N_HID), b1=g["b1"], w2=g["w2"].reshape(N_HID, N_HID), b2=g["b2"],
                w3=g["w3"].reshape(N_HID, N_HID), b3=g["b3"], w4=g["w4"].reshape(N_HID, N_OUT), b4=g["b4"])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(p, feat, emulate_bf16=True):
    q = unpack(p)
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    inv_sd = np.float32(1.0) / np.asarray(q["sd_in"], np.float32)
    x0 = r((np.asarray(feat, np.float32) - np.asarray(q["mu_in"], np.float32)) * inv_sd)
    ws = [r(q["w1"]), r(q["w2"]), r(q["w3"]), r(q["w4"])]
    bs = [q["b1"], q["b2"], q["b3"], q["b4"]]
    acts, pre = [x0], []
    a = x0
    for l in range(3):
        z = a @ ws[l] + bs[l]
        pre.append(z)
        a = r(gelu(z))
        acts.append(a)
    y = a @ ws[3] + bs[3]
    return y, acts, pre, ws


def predict(p, feat):
    q = unpack(p)
    y, _, _, _ = forward(p, feat)
    return y * q["sd_out"] + q["mu_out"]


def loss_and_grad(p, feat, target, emulate_bf16=True):
    """Loss = mean over rows and outputs of the squared error of the
    standardised output; gradient in the flat layout (normalisation zero)."""
    q = unpack(p)
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float64))
    y, acts, pre, ws = forward(p, feat, emulate_bf16)
    rows = y.shape[0]
    t = (np.asarray(target, np.float64) - q["mu_out"]) / q["sd_out"]
    d = y - t
    loss = float(np.mean(d * d))
    dz = r(d * (2.0 / (3.0 * rows)))
    grads = {}
    for l in (3, 2, 1, 0):
        grads[f"w{l + 1}"] = acts[l].T @ dz
        grads[f"b{l + 1}"] = dz.sum(0)
        if l > 0:
            da = dz @ ws[l].T
            dz = r(da * gelu_grad(pre[l - 1]))
    g = np.zeros(OFF["total"])
    for k, v in grads.items():
        a, b = OFF[k]
        g[a:b] = v.ravel()
    return loss, g


def init_params(rng, mu_in, sd_in, mu_out, sd_out):
    """He-style initialisation with the given standardisation statistics."""
    p = np.zeros(OFF["total"], np.float32)
    for k, v in (("mu_in", mu_in), ("sd_in", sd_in), ("mu_out", mu_out), ("sd_out", sd_out)):
        a, b = OFF[k]
        p[a:b] = v
    for k, fan_in, shape in (("w1", N_IN, (N_IN, N_HID)), ("w2", N_HID, (N_HID, N_HID)),
                             ("w3", N_HID, (N_HID, N_HID)), ("w4", N_HID, (N_HID, N_OUT))):
        a, b = OFF[k]
        p[a:b] = (rng.standard_normal(shape) * np.sqrt(2.0 / fan_in)).ravel()
    return p
