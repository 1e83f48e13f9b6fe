"""FP64 numpy restatement of the path-guiding network (encoding, forward,
vMF mixture, loss gradient by backpropagation, Adam).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA guide (BF16 tensor-core
kernels with FP32 accumulation); the product never imports it.  The network
has no counterpart in the reference renderer; its definition is the one in
include/lucid_cuda.h (lucid_guide_*).
"""
from __future__ import annotations

import numpy as np

N_IN, N_IN_USED, N_HID, N_OUT, LOBES, FREQ, BINS = 176, 163, 64, 48, 8, 16, 32
KAPPA_MIN, KAPPA_MAX = 0.05, 2000.0
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("W4", (N_OUT, N_HID)), ("b4", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], np.float64).ravel() for name, _ in SHAPES])


def encode(p01, n, wo):
    p01, n, wo = (np.asarray(a, np.float64).reshape(-1, 3) for a in (p01, n, wo))
    m = len(p01)
    x = np.zeros((m, N_IN))
    f = np.pi * (2.0 ** np.arange(FREQ))
    for a in range(3):
        arg = p01[:, a:a + 1] * f[None, :]
        x[:, a * 2 * FREQ:(a + 1) * 2 * FREQ:2] = np.sin(arg)
        x[:, a * 2 * FREQ + 1:(a + 1) * 2 * FREQ:2] = np.cos(arg)
    x[:, 96:99] = n
    u = np.clip(0.5 * (wo[:, 2] + 1.0), 0.0, 1.0)
    v = np.arctan2(wo[:, 1], wo[:, 0]) / (2.0 * np.pi) + 0.5
    c = (np.arange(BINS) + 0.5) / BINS
    x[:, 99:99 + BINS] = np.exp(-0.5 * ((u[:, None] - c[None, :]) * BINS) ** 2)
    x[:, 99 + BINS:99 + 2 * BINS] = np.exp(-0.5 * ((v[:, None] - c[None, :]) * BINS) ** 2)
    return x


def forward(theta, x):
    P = unpack(theta)
    z1 = x @ P["W1"].T + P["b1"]; h1 = np.maximum(z1, 0)
    z2 = h1 @ P["W2"].T + P["b2"]; h2 = np.maximum(z2, 0)
    z3 = h2 @ P["W3"].T + P["b3"]; h3 = np.maximum(z3, 0)
    raw = h3 @ P["W4"].T + P["b4"]
    return raw, (x, h1, h2, h3)


def softplus(x):
    return np.where(x > 20, x, np.log1p(np.exp(np.minimum(x, 20))))


def mixture(raw):
    logits = raw[:, :LOBES]
    w = np.exp(logits - logits.max(axis=1, keepdims=True))
    w /= w.sum(axis=1, keepdims=True)
    k = np.minimum(softplus(raw[:, LOBES:2 * LOBES]) + KAPPA_MIN, KAPPA_MAX)
    m = raw[:, 16:40].reshape(-1, LOBES, 3)
    l = np.linalg.norm(m, axis=2, keepdims=True)
    mu = np.where(l > 1e-6, m / np.maximum(l, 1e-300), np.array([0.0, 0.0, 1.0]))
    return w, k, mu


def vmf_pdf(k, mu, wi):
    """k: (m, L), mu: (m, L, 3), wi: (m, 3) -> (m, L)."""
    c = np.einsum("mlc,mc->ml", mu, wi)
    return k / (2 * np.pi * (1 - np.exp(-2 * k))) * np.exp(k * (c - 1))


def mixture_pdf(raw, wi):
    w, k, mu = mixture(raw)
    return (w * vmf_pdf(k, mu, np.asarray(wi, np.float64))).sum(axis=1)


def sample(raw, u0, u1, u2):
    """Directions drawn like the CUDA guide (lobe by u0, vMF by u1, u2)."""
    w, k, mu = mixture(raw)
    cw = np.cumsum(w, axis=1)
    lobe = np.minimum((u0[:, None] >= cw).sum(axis=1), LOBES - 1)
    idx = np.arange(len(raw))
    kk, m = k[idx, lobe], mu[idx, lobe]
    c = np.clip(1 + np.log(u1 + (1 - u1) * np.exp(-2 * kk)) / kk, -1, 1)
    r = np.sqrt(np.maximum(0, 1 - c * c))
    t, b = onb(m)
    d = t * (r * np.cos(2 * np.pi * u2))[:, None] + b * (r * np.sin(2 * np.pi * u2))[:, None] + m * c[:, None]
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def onb(n):
    """The renderer's orthonormal basis (Frisvad's construction with the
    n.z = -1 special case)."""
    a = 1.0 / (1.0 + np.where(n[:, 2] < -0.9999, 0.0, n[:, 2]))
    bb = -n[:, 0] * n[:, 1] * a
    t = np.stack([1 - n[:, 0] ** 2 * a, bb, -n[:, 0]], axis=1)
    b = np.stack([bb, 1 - n[:, 1] ** 2 * a, -n[:, 1]], axis=1)
    low = n[:, 2] < -0.9999
    t[low] = [0.0, -1.0, 0.0]
    b[low] = [-1.0, 0.0, 0.0]
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b /= np.linalg.norm(b, axis=1, keepdims=True)
    return t, b


def coefficients(recs):
    L = recs[:, 13:16]
    F = 0.2126 * L[:, 0] + 0.7152 * L[:, 1] + 0.0722 * L[:, 2]
    pdf = recs[:, 12]
    ok = (F > 0) & (pdf > 0) & np.isfinite(F)
    c = np.where(ok, F / np.where(ok, pdf, 1.0), 0.0)
    s = c.sum()
    return c / s if s > 0 else c


def loss(theta, recs):
    recs = np.asarray(recs, np.float64)
    x = encode(recs[:, 0:3], recs[:, 3:6], recs[:, 6:9])
    raw, _ = forward(theta, x)
    q = mixture_pdf(raw, recs[:, 9:12])
    c = coefficients(recs)
    return float(-(c * np.log(np.maximum(q, 1e-300))).sum())


def gradient(theta, recs, bf16_inputs=False):
    """d loss / d theta by backpropagation (records: (m, 16)); with
    bf16_inputs the encoded inputs are rounded to BF16 first, as the CUDA
    kernels feed them to the tensor cores."""
    recs = np.asarray(recs, np.float64)
    P = unpack(theta)
    x = encode(recs[:, 0:3], recs[:, 3:6], recs[:, 6:9])
    if bf16_inputs:
        x = bf16_round(x)
    raw, (x, h1, h2, h3) = forward(theta, x)
    wi = recs[:, 9:12]
    c = coefficients(recs)
    w, k, mu = mixture(raw)
    p = vmf_pdf(k, mu, wi)
    q = (w * p).sum(axis=1, keepdims=True)
    gam = w * p / np.maximum(q, 1e-300)
    d = np.zeros_like(raw)
    cc = c[:, None]
    d[:, :LOBES] = cc * (w - gam)
    e = np.exp(-2 * k)
    mw = np.einsum("mlc,mc->ml", mu, wi)
    dlogp = 1 / k - 2 * e / (1 - e) + (mw - 1)
    r = raw[:, LOBES:2 * LOBES]
    d[:, LOBES:2 * LOBES] = np.where(k < KAPPA_MAX, -cc * gam * dlogp / (1 + np.exp(-r)), 0.0)
    m = raw[:, 16:40].reshape(-1, LOBES, 3)
    l = np.linalg.norm(m, axis=2)
    gdir = (wi[:, None, :] - mu * mw[:, :, None]) * (-cc * gam * k / np.maximum(l, 1e-300))[:, :, None]
    gdir = np.where((l > 1e-6)[:, :, None], gdir, 0.0)
    d[:, 16:40] = gdir.reshape(-1, 24)
    G = {"W4": d.T @ h3, "b4": d.sum(0)}
    d3 = (d @ P["W4"]) * (h3 > 0)
    G["W3"], G["b3"] = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ P["W3"]) * (h2 > 0)
    G["W2"], G["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ P["W2"]) * (h1 > 0)
    G["W1"], G["b1"] = d1.T @ x, d1.sum(0)
    return pack(G)


def adam(theta, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    g = np.where(np.isfinite(g), g, 0.0)
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    theta = theta - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return theta, m, v


def bf16_round(a):
    """Round FP32 values to BF16 (round to nearest even), returned as FP64."""
    a = np.asarray(a, np.float32).copy()
    u = a.view(np.uint32)
    u += 0x7FFF + ((u >> 16) & 1)
    u &= 0xFFFF0000
    return u.view(np.float32).astype(np.float64)


def bf16_weights(theta):
    """theta with its weight matrices (not the biases) rounded to BF16: the
    network the CUDA kernels evaluate."""
    t = np.asarray(theta, np.float64).copy()
    o = 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        if name.startswith("W"):
            t[o:o + n] = bf16_round(t[o:o + n])
        o += n
    return t


def coherent_records(rng, n, spread=0.3):
    """Records whose sampled directions cluster around one direction: a
    well-conditioned gradient (the samples agree) for precision checks."""
    recs = random_records(rng, n)
    d0 = np.array([0.3, -0.5, 0.81])
    w = d0 / np.linalg.norm(d0) + spread * rng.normal(size=(n, 3))
    recs[:, 9:12] = w / np.linalg.norm(w, axis=1, keepdims=True)
    recs[:, 13:16] = 1.0
    return recs


def random_records(rng, n, raw_like=None):
    """Synthetic training records: positions in [0,1]^3, unit normals,
    outgoing and sampled directions, positive pdfs and radiance."""
    def unit(k):
        a = rng.normal(size=(k, 3))
        return a / np.linalg.norm(a, axis=1, keepdims=True)
    recs = np.zeros((n, 16))
    recs[:, 0:3] = rng.random((n, 3))
    recs[:, 3:6] = unit(n)
    recs[:, 6:9] = unit(n)
    recs[:, 9:12] = unit(n)
    recs[:, 12] = rng.uniform(0.05, 2.0, n)
    recs[:, 13:16] = rng.exponential(1.0, (n, 3)) * (rng.random((n, 1)) < 0.8)
    return recs
