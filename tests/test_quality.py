"""Converged FP64 references and relMSE.

CPU: the metric's definition and the oracle's FP64 accumulation (the same
per-sample values as its FP32 render, summed in double).  GPU: the CUDA FP64
accumulation equals the oracle's bit for bit on the Cornell box (the C1
reference cross-check), and error falls with samples as 1/spp."""
from __future__ import annotations

import numpy as np
import pytest

import lucid_quality as lq
import lucid_scenes as ls


def test_relmse_definition():
    ref = np.array([[[1.0, 0.0, 2.0]]])
    img = np.array([[[1.5, 0.1, 2.0]]])
    expect = (0.25 / (1.0 + 1e-2) + 0.01 / 1e-2 + 0.0) / 3.0
    assert lq.relmse(img, ref) == pytest.approx(expect, rel=1e-12)
    assert lq.relmse(ref, ref) == 0.0
    rgba = np.concatenate([img, np.ones((1, 1, 1))], axis=-1)
    assert lq.relmse(rgba, ref) == pytest.approx(expect, rel=1e-12)   # alpha ignored
    with pytest.raises(ValueError):
        lq.relmse(np.zeros((2, 2, 3)), np.zeros((2, 3, 3)))


def _cornell_oracle():
    from oracle_ctypes import Oracle
    scene, cam = ls.cornell_box()
    o = Oracle(device_math=True, canonical_ties=True)
    assert o.load_scene_json(ls.to_json(scene))
    o.set_camera(*cam)
    o.set_algorithm("mis")
    return o


def test_oracle_f64_accumulates_the_fp32_samples(oracle_lib):
    o = _cornell_oracle()
    tile = dict(tile_x=112, tile_y=100, full_w=256, full_h=256)
    img32, recs, rc = o.render(16, 8, samples=8, max_depth=8, records=True, **tile)
    assert rc == 0
    img64, rc = o.render_f64(16, 8, samples=8, max_depth=8, **tile)
    assert rc == 0
    # the same per-sample FP32 values, summed in double in sample order
    per = recs["rgb"].reshape(8, 16, 8, 3).astype(np.float64)      # [y, x, s, c]
    acc = np.zeros((8, 16, 3))
    for s in range(8):
        acc += per[:, :, s]
    np.testing.assert_array_equal(img64[::-1, :, :3], np.maximum(acc, 0.0))
    np.testing.assert_allclose(img64[..., :3], img32[..., :3], rtol=1e-5, atol=1e-6)
    one64, _ = o.render_f64(16, 8, samples=1, **tile)
    one32, _, _ = o.render(16, 8, samples=1, **tile)
    np.testing.assert_array_equal(one64, one32.astype(np.float64))


def test_oracle_error_falls_with_samples(oracle_lib):
    """relMSE against an independent 1024-spp FP64 reference falls with the
    sample count (C1 framing, a 48x48 crop of the 256x256 frame; relMSE of
    a few samples is heavy-tailed, so the fall is slower than 1/spp here)."""
    o = _cornell_oracle()
    tile = dict(tile_x=64, tile_y=64, full_w=256, full_h=256, max_depth=8)
    ref = lq.mean_image(o.render_f64(48, 48, samples=1024, sample_offset=100000, **tile)[0], 1024)
    errs = []
    for spp in (4, 16, 64):
        img = lq.mean_image(o.render_f64(48, 48, samples=spp, **tile)[0], spp)
        errs.append(lq.relmse(img, ref))
    assert errs[0] > errs[1] > errs[2] > 0
    assert errs[0] / errs[2] > 3.0


@pytest.fixture(scope="module")
def cornell_ctx():
    import lucid_capi
    scene, cam = ls.cornell_box()
    c = lucid_capi.Context(0)
    c.load_scene_json(ls.to_json(scene))
    c.set_camera(*cam)
    c.set_algorithm("mis")
    yield c
    c.close()


@pytest.mark.gpu
def test_gpu_f64_equals_oracle_f64(cornell_ctx, oracle_lib):
    """The C1 reference cross-check: GPU FP64 accumulation vs the oracle's."""
    o = _cornell_oracle()
    for spp, tile in ((64, (96, 96, 32, 24)), (4096, (124, 40, 8, 6))):
        tx, ty, tw, th = tile
        g = cornell_ctx.render_f64(tw, th, 256, 256, spp, 0, 8, tile_x=tx, tile_y=ty)
        c, rc = o.render_f64(tw, th, 256, 256, samples=spp, max_depth=8, tile_x=tx, tile_y=ty)
        assert rc == 0
        np.testing.assert_array_equal(g, c)


@pytest.mark.gpu
def test_gpu_reference_and_error_curve(cornell_ctx):
    ref = lq.render_reference(cornell_ctx, 256, 256, spp=4096, max_depth=8, sample_offset=1 << 20)
    assert ref.shape == (256, 256, 3) and np.all(np.isfinite(ref)) and ref.mean() > 0
    img32 = cornell_ctx.render(256, 256, 256, 256, 16, 0, 8)[0]
    img64 = cornell_ctx.render_f64(256, 256, 256, 256, 16, 0, 8)
    np.testing.assert_allclose(img32[..., :3], img64[..., :3], rtol=1e-5, atol=1e-5)
    e = [lq.relmse(lq.mean_image(cornell_ctx.render_f64(256, 256, 256, 256, s, 0, 8), s), ref) for s in (4, 16, 64)]
    assert e[0] > e[1] > e[2] > 0
    assert e[0] / e[2] > 3.0
