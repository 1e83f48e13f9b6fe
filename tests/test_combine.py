"""Concurrent small renders of several contexts combined into batches
(lucid_cuda_set_combining, on by default): sessions on different scenes
render from their own threads at the same time, as the add-on's viewport,
material previews and F12 renders do, and every call's image must be bit
for bit the one the same call gives alone, whether it ran on its own
context or inside a batch with the others; calls of other integrators and
calls too large to combine are not batched with them."""
from __future__ import annotations

import threading

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from parity_util import ATOL, RTOL, render_oracle, scene_and_camera


def test_combining_calls_without_a_gpu():
    lib = lucid_capi.load_library()
    assert lib.lucid_cuda_set_combining(None, 1) == lucid_capi.LUCID_ERR_INVALID
    ctx = lucid_capi.Context(0)
    ctx.set_combining(False)
    ctx.set_combining(True)
    b, c = lucid_capi.combine_stats(0)
    assert b >= 0 and c >= 0
    ctx.close()


SESSIONS = [  # scene, integrator, calls as (width, height, samples, sample offset)
    ("cornell", "mis", [(96, 96, 8, 0), (64, 48, 4, 8), (80, 60, 2, 12), (96, 96, 8, 14)]),
    ("procedural_small", "mis", [(72, 72, 6, 0), (96, 64, 3, 6), (40, 40, 16, 9), (72, 72, 6, 25)]),
    ("all_lights_novol", "mis", [(64, 64, 8, 0), (64, 64, 8, 8), (32, 24, 1, 16), (64, 64, 8, 17)]),
    ("textured", "mis", [(80, 80, 4, 0), (80, 80, 4, 4), (80, 80, 4, 8), (80, 80, 4, 12)]),
    ("mirror", "nee", [(64, 64, 8, 0), (48, 48, 4, 8), (64, 64, 8, 12), (64, 64, 8, 20)]),
    ("cornell", "mis", [(1024, 1024, 8, 100)]),   # 8.4 M paths: above the combining limit
]


def _contexts(workdir):
    out = []
    for name, algo, _ in SESSIONS:
        scene, cam = scene_and_camera(name, workdir)
        ctx = lucid_capi.Context(0)
        ctx.load_scene_json(ls.to_json(scene))
        ctx.set_camera(*cam)
        ctx.set_algorithm(algo)
        out.append(ctx)
    return out


def _render_all(ctx, calls, rounds):
    imgs = []
    for _ in range(rounds):
        for (w, h, spp, off) in calls:
            img, _, _ = ctx.render(w, h, w, h, spp, off, 8)
            imgs.append(img)
    return imgs


@pytest.mark.gpu
def test_concurrent_sessions_equal_their_calls_alone(workdir):
    ctxs = _contexts(workdir)
    rounds = 3
    # each session alone, one call after another, combining off
    for c in ctxs:
        c.set_combining(False)
    want = [_render_all(c, s[2], 1) for c, s in zip(ctxs, SESSIONS)]
    for c in ctxs:
        c.set_combining(True)
    b0, c0 = lucid_capi.combine_stats(0)
    got = [None] * len(ctxs)
    errors = []
    start = threading.Barrier(len(ctxs))

    def session(k):
        try:
            start.wait()
            got[k] = _render_all(ctxs[k], SESSIONS[k][2], rounds)
        except Exception as e:   # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=session, args=(k,)) for k in range(len(ctxs))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    b1, c1 = lucid_capi.combine_stats(0)
    for k, (name, algo, calls) in enumerate(SESSIONS):
        for r in range(rounds):
            for i in range(len(calls)):
                np.testing.assert_array_equal(got[k][r * len(calls) + i], want[k][i],
                                              err_msg="%s %s call %d round %d" % (name, algo, i, r))
    # 21 small calls per round over five threads: some ran inside batches
    assert b1 - b0 >= 1 and c1 - c0 >= 2 * (b1 - b0)
    # and directly against the CPU oracle: the first Cornell call of every round
    scene, cam = scene_and_camera("cornell", workdir)
    ref, _ = render_oracle(scene, cam, "mis", 96, 96, 8, 8, offset=0)
    for r in range(rounds):
        np.testing.assert_allclose(got[0][r * len(SESSIONS[0][2])], ref, rtol=RTOL, atol=ATOL)
    for c in ctxs:
        c.close()


@pytest.mark.gpu
def test_combined_call_reports_its_own_paths(workdir):
    """After a call that ran in a batch, the context's statistics give
    that call's path count."""
    ctxs = _contexts(workdir)[:2]
    start = threading.Barrier(2)
    stats = [None, None]

    def session(k):
        start.wait()
        for _ in range(20):
            ctxs[k].render(64, 64, 64, 64, 4, 0, 8)
        stats[k] = ctxs[k].stats()

    threads = [threading.Thread(target=session, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for s in stats:
        assert s["paths"] == 64 * 64 * 4
    for c in ctxs:
        c.close()
