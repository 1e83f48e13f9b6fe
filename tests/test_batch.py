"""Batched jobs: jobs on different scenes, cameras, image sizes and sample
counts rendered in one set of wavefront launches over a device job table
(lucid_cuda_render_batch, and the request loop's batches).  Every job's
image must be bit for bit the single render call of the same parameters on
its own scene, whatever the batch around it and however its samples are cut
across waves; one batch is also checked against the CPU oracle directly."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from parity_util import ATOL, RTOL, render_oracle, scene_and_camera


def _context(workdir, name):
    scene, cam = scene_and_camera(name, workdir)
    ctx = lucid_capi.Context(0)
    ctx.load_scene_json(ls.to_json(scene))
    return ctx, cam


def _moved(cam, dx):
    c = list(cam)
    c[0] += dx
    return tuple(c)


def _single(ctx, cam, algo, job):
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    w, h = job["width"], job["height"]
    img, _, _ = ctx.render(w, h, job.get("full_w", w), job.get("full_h", h), job.get("samples", 1),
                           job.get("sample_offset", 0), job.get("max_depth", 8), tile_x=job.get("tile_x", 0),
                           tile_y=job.get("tile_y", 0))
    return img


def test_batch_rejects_bad_jobs_without_a_gpu():
    lib = lucid_capi.load_library()
    ctx = lucid_capi.Context(0)   # no scene loaded: creating a context touches no device
    assert lib.lucid_cuda_render_batch(ctx.h, None, 0, b"mis") == lucid_capi.LUCID_ERR_INVALID
    assert lib.lucid_cuda_render_batch(None, None, 1, b"mis") == lucid_capi.LUCID_ERR_INVALID
    job = {"scene": ctx, "camera": (0, 0, 3, 0, 0, -1, 0, 1, 0, 45), "width": 4, "height": 4}
    # the binding hands the library non-zero buffers here: a refused batch
    # must leave every image zero
    arr = (lucid_capi.BatchJob * 2)()
    imgs = [np.full((4, 4, 4), 7.0, np.float32), np.full((2, 3, 4), 7.0, np.float32)]
    for k, img in enumerate(imgs):
        arr[k].scene = ctx.h
        arr[k].params = lucid_capi.RenderParams(0, 0, img.shape[1], img.shape[0], img.shape[1], img.shape[0],
                                                1, 0, 8, 0)
        arr[k].out_rgba = img.ctypes.data
    assert lib.lucid_cuda_render_batch(ctx.h, ctypes.addressof(arr), 2, b"mis") == lucid_capi.LUCID_ERR_NO_SCENE
    assert not any(img.any() for img in imgs)
    _, rc = ctx.render_batch([job], check=False)
    assert rc == lucid_capi.LUCID_ERR_NO_SCENE
    ctx.close()


CASES = {
    # integrator: jobs as (scene, camera shift, width, height, samples, sample offset, tile)
    "mis": [("cornell", 0.0, 48, 36, 4, 0, None),
            ("procedural_small", 0.0, 40, 40, 3, 5, None),
            ("cornell", 0.12, 33, 17, 1, 0, None),            # another camera on the same scene, one sample
            ("textured", 0.0, 32, 24, 2, 0, None),
            ("two_small_quads", 0.0, 20, 20, 5, 2, None),
            ("empty_env", 0.0, 8, 8, 2, 0, None),
            ("cornell", 0.0, 24, 20, 6, 9, (40, 30, 24, 20, 128, 96))],   # a tile of a larger frame
    "volume_mis": [("all_lights", 0.0, 40, 30, 3, 0, None),
                   ("two_volumes", 0.0, 36, 28, 2, 4, None),
                   ("cornell", 0.0, 30, 30, 4, 0, None)],
    "nee": [("all_lights_novol", 0.0, 32, 24, 4, 0, None),
            ("mirror", 0.0, 28, 28, 3, 1, None)],
}


def _jobs(workdir, algo, ctxs):
    jobs, cams = [], []
    for name, dx, w, h, spp, off, tile in CASES[algo]:
        if name not in ctxs:
            ctxs[name] = _context(workdir, name)
        ctx, cam = ctxs[name]
        cam = _moved(cam, dx)
        j = {"scene": ctx, "camera": cam, "width": w, "height": h, "samples": spp, "sample_offset": off,
             "max_depth": 8}
        if tile:
            j.update(tile_x=tile[0], tile_y=tile[1], width=tile[2], height=tile[3], full_w=tile[4], full_h=tile[5])
        jobs.append(j)
        cams.append(cam)
    return jobs, cams


@pytest.mark.gpu
@pytest.mark.parametrize("algo", sorted(CASES))
def test_batch_equals_single_render_calls(workdir, algo):
    ctxs = {}
    jobs, cams = _jobs(workdir, algo, ctxs)
    want = [_single(ctxs[c[0]][0], cam, algo, j) for c, cam, j in zip(CASES[algo], cams, jobs)]
    runner = lucid_capi.Context(0)   # renders the batch with its own path pool; it has no scene of its own
    got, _ = runner.render_batch(jobs, algo)
    for k in range(len(jobs)):
        np.testing.assert_array_equal(got[k], want[k], err_msg="job %d (%s)" % (k, CASES[algo][k][0]))
    # small waves: jobs split across waves in sample order, pieces of
    # several jobs in one wave; the images must not change
    largest = max(j["width"] * j["height"] for j in jobs)
    runner.set_wave_capacity(largest + 7)
    got_small, _ = runner.render_batch(jobs, algo)
    assert runner.stats()["waves"] > 4
    for k in range(len(jobs)):
        np.testing.assert_array_equal(got_small[k], want[k], err_msg="small waves, job %d" % k)
    # the rendering context may also be one of the scene contexts, and a
    # second call reuses its pool
    first = ctxs[CASES[algo][0][0]][0]
    again, _ = first.render_batch(jobs, algo)
    for k in range(len(jobs)):
        np.testing.assert_array_equal(again[k], want[k])
    runner.close()
    for c, _ in ctxs.values():
        c.close()


@pytest.mark.gpu
def test_batch_matches_the_oracle(workdir):
    """Two jobs on two scenes in one batch, each image against the CPU
    oracle's render of its own scene (per-pixel FP32 sums in sample order)."""
    ctxs = {}
    spec = [("cornell", 24, 24, 2, 0), ("procedural_small", 20, 16, 3, 7)]
    jobs = []
    for name, w, h, spp, off in spec:
        ctxs[name] = _context(workdir, name)
        jobs.append({"scene": ctxs[name][0], "camera": ctxs[name][1], "width": w, "height": h, "samples": spp,
                     "sample_offset": off, "max_depth": 8})
    got, _ = ctxs["cornell"][0].render_batch(jobs, "mis")
    for (name, w, h, spp, off), img in zip(spec, got):
        scene, cam = scene_and_camera(name, workdir)
        ref, _ = render_oracle(scene, cam, "mis", w, h, spp, 8, offset=off)
        np.testing.assert_allclose(img, ref, rtol=RTOL, atol=ATOL, err_msg=name)
    for c, _ in ctxs.values():
        c.close()


@pytest.mark.gpu
def test_batch_rejects_mixed_depths(workdir):
    ctx, cam = _context(workdir, "cornell")
    jobs = [{"scene": ctx, "camera": cam, "width": 8, "height": 8, "max_depth": 8},
            {"scene": ctx, "camera": cam, "width": 8, "height": 8, "max_depth": 4}]
    _, rc = ctx.render_batch(jobs, "mis", check=False)
    assert rc == lucid_capi.LUCID_ERR_INVALID
    ctx.close()


@pytest.mark.gpu
def test_server_batches_equal_single_render_calls(workdir):
    """Throughput jobs submitted together run as batches (the stats count
    them); their images equal single render calls, as do those of the
    server with batching off and of a job too large for a batch."""
    spec = [("cornell", 64, 48, 8), ("procedural_small", 48, 48, 4), ("all_lights_novol", 40, 30, 6),
            ("cornell", 32, 32, 16), ("procedural_small", 96, 64, 2), ("textured", 40, 40, 4)]
    names = sorted({s[0] for s in spec})
    want = []
    for name, w, h, spp in spec:
        ctx, cam = _context(workdir, name)
        want.append(_single(ctx, cam, "mis", {"width": w, "height": h, "samples": spp}))
        ctx.close()
    scenes = {n: scene_and_camera(n, workdir) for n in names}
    # 2^26: every job after the first (which starts alone, before the others
    # are queued) fits one batch; 40,000 paths: a batch of some jobs, the
    # others too large for what is left of it run on their own; 0: off
    for batching in (1 << 26, 40_000, 0):
        srv = lucid_capi.Server(0, slots=1)
        srv.set_batching(batching)
        ids = {n: srv.add_scene(ls.to_json(scenes[n][0])) for n in names}
        jids = [srv.submit(ids[n], scenes[n][1], w, h, spp, 8, "mis") for n, w, h, spp in spec]
        for j in jids:
            assert srv.wait(j, 60000) == lucid_capi.JOB_DONE
        got = [srv.result(j) for j in jids]
        st = srv.stats()
        srv.close()
        for k in range(len(spec)):
            np.testing.assert_array_equal(got[k], want[k], err_msg="batching %d, job %d" % (batching, k))
        if batching == 0:
            assert st["batches"] == 0
        else:
            assert st["batches"] >= 1 and st["batched_jobs"] >= 2
        assert st["done"] == len(spec) and st["bytes_running"] == 0
