"""The request loop: admission by device-memory budget (host-side policy,
no GPU) and, on the GPU, jobs whose images are the same alone and in a mix
of concurrent jobs, bit for bit, and equal to one render call with all
their samples."""
from __future__ import annotations

import time

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from parity_util import scene_and_camera


def test_admission_refuses_jobs_that_never_fit():
    assert lucid_capi.admission_plan(100, 20, 2, [30, 30, 50, 90, 10]) == [0, 1, 2, -1, 3]
    assert lucid_capi.admission_plan(100, 0, 4, [101, 100, 1]) == [-1, 0, 1]
    assert lucid_capi.admission_plan(10, 10, 1, [1]) == [-1]


def test_admission_is_first_come_first_served_within_slots_and_budget():
    # 3 slots, room for two 40-byte jobs at a time: arrival order is kept
    assert lucid_capi.admission_plan(100, 20, 3, [40, 40, 40, 5, 40]) == [0, 1, 2, 3, 4]
    # one slot: strictly sequential
    assert lucid_capi.admission_plan(1 << 40, 0, 1, [1, 2, 3]) == [0, 1, 2]
    assert lucid_capi.admission_plan(100, 0, 2, []) == []


def _job(w, h, spp, algo="mis", depth=8, interactive=0, guided=0):
    return {"width": w, "height": h, "samples": spp, "algorithm": algo, "max_depth": depth,
            "interactive": interactive, "guided": guided}


def test_batch_plan_takes_compatible_jobs_in_queue_order():
    big_room = 1 << 40
    head = _job(64, 64, 4)
    queue = [_job(32, 32, 8), _job(32, 32, 8, algo="nee"), _job(16, 16, 4, depth=6), _job(8, 8, 1, interactive=1),
             _job(8, 8, 1, guided=1), _job(48, 48, 2)]
    # other integrators, other depths, interactive and guided jobs stay queued
    assert lucid_capi.batch_plan(1 << 25, big_room, [head] + queue) == [1, 1, 0, 0, 0, 0, 1]
    # cancelled jobs are skipped
    assert lucid_capi.batch_plan(1 << 25, big_room, [head] + queue, [0, 1, 0, 0, 0, 0, 0]) == [1, 0, 0, 0, 0, 0, 1]
    # nothing compatible behind it: the head runs alone
    assert lucid_capi.batch_plan(1 << 25, big_room, [head, _job(8, 8, 1, algo="simple")]) == [0, 0]
    # batching off, an interactive or guided head, or a head at the path limit: alone
    assert lucid_capi.batch_plan(0, big_room, [head] + queue) == [0] * 7
    assert lucid_capi.batch_plan(1 << 25, big_room, [_job(64, 64, 4, interactive=1)] + queue) == [0] * 7
    assert lucid_capi.batch_plan(1 << 25, big_room, [_job(64, 64, 4, guided=1)] + queue) == [0] * 7
    assert lucid_capi.batch_plan(64 * 64 * 4, big_room, [head] + queue) == [0] * 7


def test_batch_plan_respects_the_path_limit_and_the_budget():
    head = _job(100, 100, 1)                      # 10,000 paths
    queue = [_job(100, 100, 3), _job(50, 50, 4), _job(100, 100, 2), _job(10, 10, 1)]
    # 40,000-path limit: 10k + 30k fits, the 10k job would exceed it, the
    # 20k job too; the last 100 paths still fit after the first
    assert lucid_capi.batch_plan(40_000, 1 << 40, [head] + queue) == [1, 1, 0, 0, 0]
    assert lucid_capi.batch_plan(40_100, 1 << 40, [head] + queue) == [1, 1, 0, 0, 1]
    # bytes: room for exactly the head and the 50x50x4 job (the 30k-path
    # job before it needs more, the 100-path job after it does not fit
    # beside them); one byte less and the 100-path job joins instead
    room = lucid_capi.batch_bytes(100 * 100 + 50 * 50, 10_000 + 10_000)
    assert lucid_capi.batch_plan(1 << 25, room, [head] + queue) == [1, 0, 1, 0, 0]
    assert lucid_capi.batch_plan(1 << 25, room - 1, [head] + queue) == [1, 0, 0, 0, 1]
    assert lucid_capi.batch_plan(1 << 25, room + 100 * (178 + 32), [head] + queue) == [1, 0, 1, 0, 1]
    # at most 256 jobs in one batch
    many = [_job(4, 4, 1)] * 300
    assert sum(lucid_capi.batch_plan(1 << 25, 1 << 40, many)) == 256


def test_server_rejects_bad_arguments_without_a_gpu():
    lib = lucid_capi.load_library()
    assert lib.lucid_server_create(0, 0, 0, None) == lucid_capi.LUCID_ERR_INVALID
    assert lib.lucid_server_submit(None, None, None) == lucid_capi.LUCID_ERR_INVALID
    assert lib.lucid_server_wait(None, 1, 0) == lucid_capi.LUCID_ERR_INVALID


JOBS = [  # scene, algorithm, width, height, samples, depth, interactive
    ("cornell", "mis", 64, 48, 16, 8, False),
    ("all_lights_novol", "nee", 80, 60, 8, 6, False),
    ("procedural_small", "mis", 96, 64, 24, 8, False),
    ("cornell", "mis", 32, 32, 64, 8, True),
    ("all_lights_novol", "mis", 40, 30, 1, 4, True),
]


def _single_call(workdir, name, algo, w, h, spp, depth):
    scene, cam = scene_and_camera(name, workdir)
    ctx = lucid_capi.Context(0)
    ctx.load_scene_json(ls.to_json(scene))
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    img, _, _ = ctx.render(w, h, w, h, spp, 0, depth)
    ctx.close()
    return img


def _submit_all(srv, ids, workdir, jobs):
    out = []
    for name, algo, w, h, spp, depth, inter in jobs:
        _, cam = scene_and_camera(name, workdir)
        out.append(srv.submit(ids[name], cam, w, h, spp, depth, algo, inter))
    return out


@pytest.mark.gpu
def test_jobs_equal_alone_in_a_mix_and_one_render_call(workdir):
    names = sorted({j[0] for j in JOBS})
    want = [_single_call(workdir, n, a, w, h, s, d) for n, a, w, h, s, d, _ in JOBS]

    alone = []
    srv = lucid_capi.Server(0, slots=1)
    ids = {n: srv.add_scene(ls.to_json(scene_and_camera(n, workdir)[0])) for n in names}
    for job in JOBS:
        jid = _submit_all(srv, ids, workdir, [job])[0]
        assert srv.wait(jid, 60000) == lucid_capi.JOB_DONE
        alone.append(srv.result(jid))
    srv.close()

    srv = lucid_capi.Server(0, slots=3)
    # this server takes its scenes as arrays: the jobs must not change
    ids = {n: srv.add_scene_arrays(ls.scene_arrays(scene_and_camera(n, workdir)[0])) for n in names}
    jids = _submit_all(srv, ids, workdir, JOBS + JOBS)   # every job twice, all at once
    for jid in jids:
        assert srv.wait(jid, 60000) == lucid_capi.JOB_DONE
    mixed = [srv.result(j) for j in jids]
    st = srv.stats()
    srv.close()

    for k in range(len(JOBS)):
        np.testing.assert_array_equal(alone[k], want[k])
        np.testing.assert_array_equal(mixed[k], want[k])
        np.testing.assert_array_equal(mixed[k + len(JOBS)], want[k])
    assert st["done"] == 2 * len(JOBS) and st["refused"] == 0
    assert st["latency_p99_ms"] >= st["latency_p50_ms"] > 0 and st["samples_per_s"] > 0
    assert st["bytes_running"] == 0


@pytest.mark.gpu
def test_budget_refusal_and_cancel(workdir):
    scene, cam = scene_and_camera("cornell", workdir)
    srv = lucid_capi.Server(0, slots=1, budget_bytes=64 << 20)
    sid = srv.add_scene(ls.to_json(scene))
    # 4096 x 4096 needs far more than 64 MB of film and path state
    big = srv.submit(sid, cam, 4096, 4096, 64, 8, "mis", check=False)
    assert srv.state(big)[0] == lucid_capi.JOB_REFUSED
    assert srv.wait(big, 0) == lucid_capi.JOB_REFUSED
    with pytest.raises(lucid_capi.LucidError):
        srv.result(big)
    long_job = srv.submit(sid, cam, 256, 256, 100000, 8, "mis")
    queued = srv.submit(sid, cam, 64, 64, 4, 8, "mis")
    time.sleep(0.2)
    srv.cancel(long_job)
    assert srv.wait(long_job, 60000) == lucid_capi.JOB_CANCELLED
    assert srv.wait(queued, 60000) == lucid_capi.JOB_DONE
    st = srv.stats()
    assert st["refused"] == 1 and st["done"] == 1
    srv.close()


@pytest.mark.gpu
def test_interactive_job_runs_between_the_iterations_of_a_long_batch_job(workdir):
    """One slot busy with a long batch render: an interactive job submitted
    meanwhile finishes well before it (it runs between the batch job's
    iterations), and both images still equal single render calls."""
    scene, cam = scene_and_camera("procedural_small", workdir)
    big = ("procedural_small", "mis", 640, 480, 1024, 8)
    small = ("procedural_small", "mis", 64, 48, 4, 8)
    srv = lucid_capi.Server(0, slots=1)
    sid = srv.add_scene(ls.to_json(scene))
    b = srv.submit(sid, cam, big[2], big[3], big[4], big[5], big[1], False)
    while srv.state(b)[0] != lucid_capi.JOB_RUNNING:
        time.sleep(0.001)
    time.sleep(0.05)
    i = srv.submit(sid, cam, small[2], small[3], small[4], small[5], small[1], True)
    assert srv.wait(i, 60000) == lucid_capi.JOB_DONE
    batch_state_when_interactive_done = srv.state(b)[0]
    assert srv.wait(b, 120000) == lucid_capi.JOB_DONE
    img_i, img_b = srv.result(i), srv.result(b)
    srv.close()
    assert batch_state_when_interactive_done == lucid_capi.JOB_RUNNING
    np.testing.assert_array_equal(img_i, _single_call(workdir, *small))
    np.testing.assert_array_equal(img_b, _single_call(workdir, *big))
