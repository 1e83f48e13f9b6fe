"""Progressive accumulator (render_*_async, pybind_renderer.hpp:689-856) on the
GPU: a snapshot after n samples equals the average of n one-sample renders
with sample offsets 0..n-1; reset wipes the accumulator; stop ends the
worker."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, DEPTH = 48, 40, 8


def _wait(pred, timeout=60.0):
    t0 = time.time()
    while time.time() - t0 < timeout:
        if pred():
            return True
        time.sleep(0.01)
    return False


def test_async_snapshot_equals_average_of_one_sample_renders():
    import lucid_capi
    import lucid_scenes as ls
    ctx = lucid_capi.Context(0)
    sc, cam = ls.cornell_box()
    ctx.load_scene_json(ls.to_json(sc))
    ctx.set_camera(*cam)
    ctx.set_algorithm("mis")
    ctx.async_start(W, H, DEPTH)
    assert ctx.async_running()
    assert _wait(lambda: ctx.async_poll()[0] >= 16)
    n, img = ctx.async_poll()
    rev = ctx.async_revision()
    ctx.async_stop()
    assert not ctx.async_running()
    assert rev >= 5   # snapshots at 1, 2, 4, 8, 16, ...
    acc = np.zeros((H, W, 4), np.float32)
    for k in range(n):
        one, _, _ = ctx.render(W, H, samples=1, sample_offset=k, max_depth=DEPTH)
        acc = acc + one
    want = acc / np.float32(n)
    want[..., 3] = 1.0
    np.testing.assert_allclose(img, want, rtol=1e-6, atol=1e-7)

    # reset wipes the accumulator: the sample count restarts
    ctx.async_start(W, H, DEPTH)
    assert _wait(lambda: ctx.async_poll()[0] >= 64)
    # calls from another thread get the GPU promptly while the worker runs
    t0 = time.time()
    ctx.set_camera(0.5, 0.5, 1.9, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 35.0)
    ctx.async_reset(W, H, DEPTH)
    assert time.time() - t0 < 2.0
    assert _wait(lambda: 0 < ctx.async_poll()[0] < 64 or ctx.async_revision() > 0)
    ctx.async_stop()
    ctx.close()


def test_pybind_async_surface():
    import lucidrenderer
    import lucid_scenes as ls
    r = lucidrenderer.Renderer()
    sc, cam = ls.cornell_box()
    assert r.load_scene_json(ls.to_json(sc))
    r.set_camera(*cam)
    r.set_algorithm("mis")
    n, px = r.render_poll_async()
    assert n == 0 and len(px) == 0
    r.render_start_async(W, H, DEPTH)
    assert r.is_render_async_running()
    assert _wait(lambda: r.render_poll_async()[0] >= 4)
    n, px = r.render_poll_async()
    assert px.shape == (W * H * 4,) and np.all(px[3::4] == 1.0) and px[0::4].sum() > 0
    assert r.render_snapshot_revision_async() >= 3
    r.render_stop_async()
    assert not r.is_render_async_running()


def test_async_snapshot_equals_the_oracle():
    """The accumulator checked against the CPU oracle directly: a snapshot
    after n samples equals the oracle's one-sample renders at sample offsets
    0..n-1, summed in order and divided by n."""
    import lucid_capi
    import lucid_scenes as ls
    from parity_util import render_oracle
    sc, cam = ls.cornell_box()
    ctx = lucid_capi.Context(0)
    ctx.load_scene_json(ls.to_json(sc))
    ctx.set_camera(*cam)
    ctx.set_algorithm("mis")
    ctx.async_start(W, H, DEPTH)
    assert _wait(lambda: ctx.async_poll()[0] >= 8)
    ctx.async_stop()
    n, img = ctx.async_poll()
    ctx.close()
    acc = np.zeros((H, W, 4), np.float32)
    for k in range(n):
        one, _ = render_oracle(sc, cam, "mis", W, H, 1, DEPTH, offset=k)
        acc = acc + one.astype(np.float32)
    want = acc / np.float32(n)
    want[..., 3] = 1.0
    np.testing.assert_allclose(img, want, rtol=1e-6, atol=1e-7)
