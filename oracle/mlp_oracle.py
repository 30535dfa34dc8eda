"""numpy restatement of the learned warm start (csrc/mlp.cu): sketch features, MLP forward and
backward, and the closed-form P step.

TEST INFRASTRUCTURE ONLY (the checker of the device kernels).  The warm start has no
counterpart in the reference, so there is nothing to pin it to beyond its own definition and
finite differences.
"""
from __future__ import annotations

import numpy as np

M64 = (1 << 64) - 1


def _mix(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def hash3(seed: int, a: int, b: int) -> int:
    """the counter hash of synth.h"""
    x = _mix((seed + 0x9E3779B97F4A7C15 * (a + 1)) & M64)
    return _mix(x ^ ((b * 0xD1B54A32D192ED03 + 0x8CB92BA72F3D8DD7) & M64))


def codes(bed: np.ndarray, I: int) -> np.ndarray:
    """2-bit codes, shape (I, J), from SNP-major packed bytes (J, ceil(I/4))."""
    J, Ib = bed.shape
    c = np.empty((J, 4 * Ib), np.uint8)
    for s in range(4):
        c[:, s::4] = (bed >> (2 * s)) & 3
    return c[:, :I].T


def sketch(bed: np.ndarray, I: int, snps: np.ndarray, R: int, seed: int):
    c = codes(bed, I)[:, snps].astype(np.int64)              # I x S
    dos = np.where(c == 1, 3, np.where(c == 0, 0, c - 1)).astype(np.int8)
    nm = dos != 3
    g = np.where(nm, dos, 0).astype(np.float64)
    freq = (g.sum(0) / np.maximum(2.0 * nm.sum(0), 1)).astype(np.float32)
    freq = np.where(nm.sum(0) > 0, freq, 0.5).astype(np.float32)
    z = np.where(nm, (g - 2.0 * freq) / np.sqrt(np.maximum(2.0 * freq * (1.0 - freq), 1e-6)), 0.0)
    S = len(snps)
    sign = np.empty((S, R))
    for s in range(S):
        h = hash3(seed, s, 0)
        for r in range(R):
            sign[s, r] = 1.0 if (h >> r) & 1 else -1.0
    proj = (z @ sign) / np.sqrt(S)
    return freq, dos, proj.astype(np.float32)


def inputs(dos, center, proj):
    x = np.where(dos == 3, 0.0, dos.astype(np.float64) - center[None, :])
    return np.concatenate([x, proj.astype(np.float64)], axis=1)


def forward(params: dict, dos, center, proj):
    x = inputs(dos, center, proj)
    h1 = np.maximum(x @ params["w1"] + params["b1"], 0.0)
    h2 = np.maximum(h1 @ params["w2"] + params["b2"], 0.0)
    z = h2 @ params["w3"] + params["b3"]
    z = z - z.max(1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(1, keepdims=True)
    return x, h1, h2, z, p


def loss_and_grads(params: dict, dos, center, proj, target):
    """mean cross-entropy against soft targets and its gradients"""
    n = dos.shape[0]
    x, h1, h2, z, p = forward(params, dos, center, proj)
    logp = z - np.log(np.exp(z).sum(1, keepdims=True))
    loss = -(target * logp).sum() / n
    dz = (p - target) / n
    g = {"w3": h2.T @ dz, "b3": dz.sum(0)}
    dh2 = (dz @ params["w3"].T) * (h2 > 0)
    g["w2"], g["b2"] = h1.T @ dh2, dh2.sum(0)
    dh1 = (dh2 @ params["w2"].T) * (h1 > 0)
    g["w1"], g["b1"] = x.T @ dh1, dh1.sum(0)
    return loss, g


def warm_p(bed, I, K, q):
    """p_kj = sum_i nm q_ki g_ij / (2 sum_i nm q_ki), clamped to [1e-5, 1-1e-5]; q is (I, K)"""
    c = codes(bed, I).astype(np.int64)
    nm = (c != 1).astype(np.float64)
    g = np.where(c == 0, 0, np.where(c == 1, 0, c - 1)).astype(np.float64)
    num = (g * nm).T @ q
    den = 2.0 * nm.T @ q
    return np.clip(np.where(den > 0, num / np.maximum(den, 1e-300), 0.5), 1e-5, 1 - 1e-5)
