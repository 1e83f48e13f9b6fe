"""The path-guiding network: the FP64 restatement's own consistency on the
CPU (backpropagation against finite differences, vMF mixture normalisation
and sampling), and on the GPU the CUDA network (BF16 tensor cores, FP32
accumulation) against that restatement: encoding, forward values, loss
gradients (relative error <= 2e-2 per parameter block) and one Adam step."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import guide_oracle as go

RTOL_BF16 = 2e-2
# The first layer's gradient passes through three BF16 backward GEMMs and is a
# sum over thousands of records with partial cancellation: ~2 % measured.
RTOL_BF16_W1 = 3e-2


def test_param_count_matches_the_library():
    import lucid_capi
    assert go.N_PARAMS == lucid_capi.load_library().lucid_guide_num_params() == 22768


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(1)
    theta = rng.normal(0, 0.2, go.N_PARAMS)
    recs = go.random_records(rng, 24)
    g = go.gradient(theta, recs)
    for idx in rng.choice(go.N_PARAMS, 40, replace=False):
        h = 1e-6
        tp, tm = theta.copy(), theta.copy()
        tp[idx] += h
        tm[idx] -= h
        fd = (go.loss(tp, recs) - go.loss(tm, recs)) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 + 1e-4 * abs(fd), idx


def test_vmf_mixture_integrates_to_one_and_sampling_follows_it():
    rng = np.random.default_rng(2)
    raw = rng.normal(0, 1.5, (1, go.N_OUT))
    n = 400000
    # uniform directions: E[q / (1 / 4 pi)] = 1
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    q = go.mixture_pdf(np.repeat(raw, n, 0), d)
    assert abs(q.mean() * 4 * np.pi - 1.0) < 0.02
    # sampled directions follow q: E_q[1 / q] = 4 pi
    s = go.sample(np.repeat(raw, n, 0), rng.random(n), rng.random(n), rng.random(n))
    inv = 1.0 / go.mixture_pdf(np.repeat(raw, n, 0), s)
    assert abs(inv.mean() / (4 * np.pi) - 1.0) < 0.03


def test_adam_restatement_first_step():
    theta = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    t, m, v = go.adam(theta, np.zeros(2), np.zeros(2), g, 1, 1e-2)
    np.testing.assert_allclose(t, theta - 1e-2 * np.sign(g), rtol=1e-6)


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def guide():
    import lucid_capi
    lib = lucid_capi.load_library()
    h = ctypes.c_void_p()
    assert lib.lucid_guide_create(0, 3, ctypes.byref(h)) == 0
    yield lib, h
    lib.lucid_guide_destroy(h)


def _params(lib, h):
    out = np.zeros(go.N_PARAMS, np.float32)
    assert lib.lucid_guide_get_params(h, out.ctypes.data, out.size) == go.N_PARAMS
    return out


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.gpu
def test_gpu_encoding_matches(guide):
    lib, h = guide
    rng = np.random.default_rng(4)
    recs = go.random_records(rng, 300).astype(np.float32)
    p, nrm, wo = (np.ascontiguousarray(recs[:, a:a + 3]) for a in (0, 3, 6))
    out = np.zeros((300, go.N_IN), np.float32)
    assert lib.lucid_guide_encode(h, p.ctypes.data, nrm.ctypes.data, wo.ctypes.data, 300, out.ctypes.data) == 0
    ref = go.encode(p, nrm, wo)
    # sin/cos of pi 2^15 x in FP32: the argument itself carries ~1e-2 rad of error
    assert np.abs(out[:, 96:] - ref[:, 96:]).max() < 1e-5
    assert np.abs(out[:, :80] - ref[:, :80]).max() < 2e-3
    assert np.abs(out[:, :96] - ref[:, :96]).max() < 5e-2


@pytest.mark.gpu
def test_gpu_forward_matches_fp64(guide):
    lib, h = guide
    rng = np.random.default_rng(5)
    theta = rng.normal(0, 0.15, go.N_PARAMS).astype(np.float32)
    assert lib.lucid_guide_set_params(h, theta.ctypes.data, theta.size) == 0
    x = go.encode(rng.random((500, 3)), rng.normal(size=(500, 3)), rng.normal(size=(500, 3))).astype(np.float32)
    out = np.zeros((500, go.N_OUT), np.float32)
    assert lib.lucid_guide_forward(h, x.ctypes.data, 500, out.ctypes.data) == 0
    ref, _ = go.forward(go.bf16_weights(theta), x.astype(np.float64))
    assert _rel(out, ref) < RTOL_BF16


@pytest.mark.gpu
def test_gpu_gradient_matches_fp64(guide):
    """Against the FP64 gradient of the network the kernels evaluate (weights
    and encoded inputs rounded to BF16; hidden activations and gradients stay
    BF16 on the GPU): relative error <= 2e-2 per parameter block (3e-2 for
    the first layer) on records
    whose samples agree, and <= 1e-1 on random records, where the gradient is
    a small sum of large cancelling terms (there even rounding the weights to
    BF16 moves the FP64 gradient by 4-6 %)."""
    lib, h = guide
    rng = np.random.default_rng(6)
    theta = rng.normal(0, 0.15, go.N_PARAMS).astype(np.float32)
    assert lib.lucid_guide_set_params(h, theta.ctypes.data, theta.size) == 0
    tq = go.bf16_weights(theta)
    for recs, tol in ((go.coherent_records(rng, 4096), RTOL_BF16), (go.random_records(rng, 4096), 0.1)):
        recs = recs.astype(np.float32)
        g = np.zeros(go.N_PARAMS, np.float32)
        assert lib.lucid_guide_gradient(h, recs.ctypes.data, len(recs), g.ctypes.data) == 0
        ref = go.gradient(tq, recs.astype(np.float64), bf16_inputs=True)
        o = 0
        for name, shape in go.SHAPES:
            n = int(np.prod(shape))
            t = max(tol, RTOL_BF16_W1) if name in ("W1", "b1") else tol
            assert _rel(g[o:o + n], ref[o:o + n]) < t, (name, t)
            o += n


@pytest.mark.gpu
def test_gpu_adam_step_matches_fp64(guide):
    lib, h = guide
    rng = np.random.default_rng(7)
    theta = rng.normal(0, 0.15, go.N_PARAMS).astype(np.float32)
    assert lib.lucid_guide_set_params(h, theta.ctypes.data, theta.size) == 0
    recs = go.random_records(rng, 2048).astype(np.float32)
    g = np.zeros(go.N_PARAMS, np.float32)
    assert lib.lucid_guide_gradient(h, recs.ctypes.data, len(recs), g.ctypes.data) == 0
    assert lib.lucid_guide_train(h, recs.ctypes.data, len(recs), ctypes.c_float(1e-2)) == 0
    after = _params(lib, h)
    want, _, _ = go.adam(theta.astype(np.float64), np.zeros(go.N_PARAMS), np.zeros(go.N_PARAMS),
                         g.astype(np.float64), 1, 1e-2)
    # FP32 against FP64 Adam: the first step is lr * g / (|g| + eps), ill
    # conditioned where |g| is near eps; 1e-4 is 1 % of the step size
    np.testing.assert_allclose(after, want, rtol=1e-5, atol=1e-4)
    # a step against its own gradient lowers the loss
    assert go.loss(after.astype(np.float64), recs) < go.loss(theta.astype(np.float64), recs)


@pytest.mark.gpu
def test_gpu_gradient_over_many_chunks_and_a_ragged_tail(guide):
    """The weight-gradient GEMMs stream 64-record chunks through a two-stage
    pipeline, several chunks per block: 65,573 records (1,025 chunks, the
    last one 37 records long and read as zeros past its end) against the FP64
    gradient, and the sum of two calls equals one call on the concatenation."""
    lib, h = guide
    rng = np.random.default_rng(8)
    theta = rng.normal(0, 0.15, go.N_PARAMS).astype(np.float32)
    assert lib.lucid_guide_set_params(h, theta.ctypes.data, theta.size) == 0
    tq = go.bf16_weights(theta)
    recs = go.coherent_records(rng, 65573).astype(np.float32)
    g = np.zeros(go.N_PARAMS, np.float32)
    assert lib.lucid_guide_gradient(h, recs.ctypes.data, len(recs), g.ctypes.data) == 0
    ref = go.gradient(tq, recs.astype(np.float64), bf16_inputs=True)
    o = 0
    for name, shape in go.SHAPES:
        n = int(np.prod(shape))
        t = RTOL_BF16_W1 if name in ("W1", "b1") else RTOL_BF16
        assert _rel(g[o:o + n], ref[o:o + n]) < t, (name, t)
        o += n
    # 37 records alone: one ragged chunk
    small = np.ascontiguousarray(recs[:37])
    gs = np.zeros(go.N_PARAMS, np.float32)
    assert lib.lucid_guide_gradient(h, small.ctypes.data, 37, gs.ctypes.data) == 0
    refs = go.gradient(tq, small.astype(np.float64), bf16_inputs=True)
    assert _rel(gs, refs) < 0.1
