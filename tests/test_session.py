"""The add-on's RenderSession and F12 loop over the CUDA module
(LucidRenderer/render_session.py:61-674, engine.py:401-447, 558-599).

The reference loop's arithmetic is restated here with the reference's own
containers (``array('f')`` and Python floats), and the numpy path must give
the same float32 values bit for bit."""
from array import array

import numpy as np
import pytest

import lucid_session as lsn


def _reference_schedule(target):
    # engine.py:558-573, written out as the reference loop runs it
    if target <= 16:
        return [target]
    out, remaining, batch = [], target, 4
    while remaining > 0:
        s = min(batch, remaining)
        out.append(s)
        remaining -= s
        batch = min(batch * 2, 64)
    return out


def _reference_accumulate(iteration_pixels):
    # engine.py:435-443: array('f') of the first result, then a per-float
    # Python loop adding every later result
    acc = None
    for px in iteration_pixels:
        if acc is None:
            acc = array("f", px)
        else:
            for i in range(len(acc)):
                acc[i] += px[i]
    return acc


def _reference_display(pixels, total):
    # engine.py:589-598: lists of [r, g, b, 1.0] scaled in double; Blender
    # keeps the Combined pass as float32
    inv = 1.0 / total
    rows = []
    for i in range(0, len(pixels), 4):
        rows.append([pixels[i] * inv, pixels[i + 1] * inv, pixels[i + 2] * inv, 1.0])
    return np.array(rows, dtype=np.float32)


@pytest.mark.parametrize("target,expected", [
    (1, [1]), (16, [16]), (17, [4, 8, 5]), (64, [4, 8, 16, 32, 4]), (128, [4, 8, 16, 32, 64, 4]),
    (300, [4, 8, 16, 32, 64, 64, 64, 48]),
])
def test_sample_schedule(target, expected):
    assert lsn.compute_sample_iterations(target) == expected == _reference_schedule(target)
    assert sum(lsn.compute_sample_iterations(target)) == target


def test_numpy_accumulate_matches_float_list_loop():
    rng = np.random.default_rng(3)
    n = 4096
    # sums spanning many binades, exact zeros and the alpha channel's 1.0s
    iters = []
    for k in range(6):
        v = (rng.random(n) * 10.0 ** rng.integers(-12, 6, n)).astype(np.float32)
        v[rng.random(n) < 0.1] = 0.0
        v[3::4] = 1.0
        iters.append(v)
    ref = np.frombuffer(_reference_accumulate([v.tolist() for v in iters]), dtype=np.float32)
    acc = iters[0].copy()
    for v in iters[1:]:
        np.add(acc, v, out=acc)
    assert np.array_equal(acc.view(np.uint32), ref.view(np.uint32))


def test_display_pixels_match_reference_conversion():
    rng = np.random.default_rng(4)
    acc = (rng.random(1024 * 4) * 10.0 ** rng.integers(-8, 5, 1024 * 4)).astype(np.float32)
    for total in (1, 3, 28, 60, 1000):
        ref = _reference_display(acc.tolist(), total)
        got = lsn.display_pixels(acc, total)
        assert got.shape == (1024, 4)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_display_pixels_on_the_host_threads_match_reference_conversion():
    """A frame larger than one host-thread chunk (ragged last chunk):
    every float of the threaded conversion, into a new array and into a
    reused one, equals the reference's per-value conversion."""
    rng = np.random.default_rng(5)
    n_px = 3 * (1 << 16) + 37          # 786,580 floats: four chunks of 2^18 floats, the last one short
    acc = (rng.random(n_px * 4) * 10.0 ** rng.integers(-8, 5, n_px * 4)).astype(np.float32)
    out = np.full(n_px * 4, np.nan, np.float32)
    for total in (3, 60):
        ref = _reference_display(acc.tolist(), total)
        for got in (lsn.display_pixels(acc, total), lsn.display_pixels(acc, total, out=out)):
            assert got.shape == (n_px, 4)
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_session_without_scene():
    s = lsn.RenderSession()
    assert s.is_available and "available" in repr(s)
    assert s.load_scene_json("{broken") is False
    # no scene / camera: a zero buffer, not cancelled (pybind_renderer.hpp:200-203)
    r = s.render_tile(lsn.RenderParams(width=6, height=4, samples=2))
    assert r.pixels.dtype == np.float32 and r.pixels.shape == (6 * 4 * 4,) and not r.pixels.any()
    assert not r.cancelled and r.job_id == 1 and r.samples == 2
    # diagnostics disabled: the reference's defaults
    assert s.get_diagnostic_stats() is None and s.export_diagnostic_json() == "{}"
    assert s.get_top_variance_groups(3) is None
    assert s.poll_render_async()[0] == 0 and s.snapshot_revision_async() == 0
    s.shutdown()
    assert not s.is_available
    r = s.render_tile(lsn.RenderParams(width=2, height=2))
    assert r.cancelled and len(r.pixels) == 0


def test_render_tile_numpy_out_checks():
    import lucidrenderer as lr
    r = lr.Renderer()
    out = np.ones(5 * 3 * 4, np.float32)
    got = r.render_tile_numpy(0, 0, 5, 3, 5, 3, out=out)
    assert got.ctypes.data == out.ctypes.data and not out.any()   # written in place (zeros: no scene)
    assert r.render_tile_numpy(0, 0, 5, 3, 5, 3).shape == (3, 5, 4)
    with pytest.raises(ValueError):
        r.render_tile_numpy(0, 0, 5, 3, 5, 3, out=np.zeros(5 * 3 * 4, np.float64))
    with pytest.raises(ValueError):
        r.render_tile_numpy(0, 0, 5, 3, 5, 3, out=np.zeros(5 * 3 * 4 - 1, np.float32))
    with pytest.raises(ValueError):
        r.render_tile_numpy(0, 0, 5, 3, 5, 3, out=np.zeros((5 * 4, 6), np.float32)[:, ::2])
    with pytest.raises(ValueError):
        r.render_tile_numpy(0, 0, 0, 3, 5, 3)


def test_f12_loop_host_logic():
    s = lsn.RenderSession()
    shown, progress = [], []
    res = lsn.render_f12(s, 8, 4, 40, on_result=lambda rect, n: shown.append((rect.shape, n)),
                         on_progress=lambda p, done, tot, eta: progress.append((done, tot)))
    assert res.iterations == [4, 8, 16, 12] and res.total_samples == 40 and not res.cancelled
    assert shown == [((32, 4), 4), ((32, 4), 12), ((32, 4), 28), ((32, 4), 40)]
    assert progress == [(0, 40), (4, 40), (12, 40), (28, 40)]
    assert res.accumulated.shape == (8 * 4 * 4,) and not res.accumulated.any()
    polls = []

    def stop_at_third_iteration():
        polls.append(1)
        return len(polls) > 2

    res = lsn.render_f12(s, 8, 4, 40, test_break=stop_at_third_iteration)
    assert res.cancelled and res.total_samples == 12 and s.is_cancelled()
    s.reset_cancel()
    s.shutdown()


# --------------------------------------------------------------------------
# On the GPU: the F12 sums against the reference's list loop and the oracle
# --------------------------------------------------------------------------

W, H = 48, 40


@pytest.mark.gpu
def test_f12_matches_list_loop_and_oracle():
    import lucid_scenes as ls
    from parity_util import RTOL, ATOL, render_oracle
    scene, cam = ls.cornell_box()
    s = lsn.RenderSession()
    assert s.load_scene_json(ls.to_json(scene))
    s.set_camera(lsn.CameraParams(pos=cam[0:3], dir=cam[3:6], up=cam[6:9], fov=cam[9]))
    res = lsn.render_f12(s, W, H, 40, max_bounces=8, algorithm="mis")
    assert res.iterations == [4, 8, 16, 12] and res.total_samples == 40 and not res.cancelled

    # the reference's loop over the list-returning method, same renderer
    r = s.renderer
    lists, offset = [], 0
    for n in res.iterations:
        lists.append(r.render_tile(0, 0, W, H, W, H, samples=n, sample_offset=offset, max_depth=8))
        offset += n
    ref = np.frombuffer(_reference_accumulate(lists), dtype=np.float32)
    assert np.array_equal(res.accumulated.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(lsn.display_pixels(res.accumulated, 40), _reference_display(ref.tolist(), 40))

    # against the oracle, iteration by iteration
    acc, offset = None, 0
    for n in res.iterations:
        img, _ = render_oracle(scene, cam, "mis", W, H, n, 8, offset=offset)
        img = np.asarray(img, np.float32).reshape(-1)
        acc = img.copy() if acc is None else acc + img
        offset += n
    np.testing.assert_allclose(res.accumulated, acc, rtol=RTOL, atol=ATOL * 40)
    s.shutdown()


@pytest.mark.gpu
def test_session_debug_and_async_paths():
    import lucid_scenes as ls
    scene, cam = ls.cornell_box()
    s = lsn.RenderSession()
    assert s.load_scene_json(ls.to_json(scene))
    # same text: no reload
    assert s.load_scene_if_changed(s._scene_hash, "{broken")
    s.set_camera_from_dict({"pos": cam[0:3], "dir": cam[3:6], "up": cam[6:9], "fov": cam[9]})
    r = s.renderer
    for mode in ("NORMAL", "albedo", "EMISSION"):
        got = s.render_tile(lsn.RenderParams(width=W, height=H, debug_mode=mode, backend="gpu"))
        want = np.asarray(r.render_debug(0, 0, W, H, W, H, mode.lower()), np.float32)
        assert np.array_equal(got.pixels, want)
    # numpy render into a reused buffer equals the list method
    out = np.empty(W * H * 4, np.float32)
    got = s.render_tile(lsn.RenderParams(width=W, height=H, samples=3, sample_offset=5, algorithm="nee"), out=out)
    assert got.pixels.ctypes.data == out.ctypes.data
    want = np.asarray(r.render_tile(0, 0, W, H, W, H, samples=3, sample_offset=5, max_depth=8), np.float32)
    assert np.array_equal(out, want)
    # the async accumulator through the session
    import time
    assert s.start_render_async(W, H, 8)
    t0 = time.time()
    while s.poll_render_async()[0] < 4 and time.time() - t0 < 20:
        time.sleep(0.01)
    n, px = s.poll_render_async()
    assert n >= 4 and px.shape == (W * H * 4,)
    s.stop_render_async()
    assert not s.is_render_async_running()
    s.shutdown()
