"""Parameter edits of an uploaded scene (lucid_cuda_update_scene,
lucid_server_update_scene) and guided jobs in the request loop.

An edited scene renders bit-identically, sample by sample, to loading the
edited scene from scratch; edits that would change the light list are
refused with nothing changed; a server job renders the scene version that
was current when it was submitted, alone or among other jobs; a guided job
(online path guiding, trained per job) is unbiased against an FP64
reference of the plain estimator, and unguided jobs beside it stay
bit-identical to single render calls.
"""
from __future__ import annotations

import copy
import time

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from parity_util import compare_records, scene_and_camera

pytestmark = pytest.mark.gpu


def _edits_and_edited_scene(scene):
    """A few edits of the all-lights scene and the same scene edited in its
    JSON form: a floor colour and roughness, the metal box's metalness (its
    shading class changes), the emissive triangle's emission (still
    emitting), a point light's energy and colour, the spot light's position,
    and the rectangle light's size (its area and so the light CDF change)."""
    edited = copy.deepcopy(scene)
    m0 = edited["meshes"][0]["material"]
    m0["base_color"] = [0.2, 0.7, 0.3]
    m0["roughness"] = 0.35
    edited["meshes"][3]["material"]["metallic"] = 0.1
    edited["meshes"][4]["material"]["emission"] = [2.0, 5.0, 9.0]
    edited["native_lights"][0]["energy"] = 250.0
    edited["native_lights"][0]["color"] = [0.4, 0.8, 1.0]
    edited["native_lights"][2]["position"] = [1.0, 2.5, 0.5]
    edited["native_lights"][5]["size"] = 1.6
    arr = ls.scene_arrays(edited)   # the values as the JSON loader reads them
    mat = lambda i: {k: arr["meshes"][i][k] for k in ("base_color", "metallic", "roughness", "emission",
                                                       "transmission", "ior")}
    edits = [{"mesh": 0, "material": mat(0)}, {"mesh": 3, "material": mat(3)}, {"mesh": 4, "material": mat(4)},
             {"light": 0, "desc": arr["lights"][0]}, {"light": 2, "desc": arr["lights"][2]},
             {"light": 5, "desc": arr["lights"][5]}]
    return edits, edited


def _ctx(scene, cam, algo):
    c = lucid_capi.Context(0)
    c.load_scene_json(ls.to_json(scene))
    c.set_camera(*cam)
    c.set_algorithm(algo)
    return c


@pytest.mark.parametrize("algo", ["mis", "volume_mis"])
def test_edited_scene_renders_as_the_edited_scene_loaded(workdir, algo):
    scene, cam = scene_and_camera("all_lights", workdir)
    edits, edited = _edits_and_edited_scene(scene)
    a = _ctx(scene, cam, algo)
    before, rb, _ = a.render(48, 36, 48, 36, 4, 1, 8, records=True)
    a.update_scene(edits)
    got, rg, _ = a.render(48, 36, 48, 36, 4, 1, 8, records=True)
    a.close()
    b = _ctx(edited, cam, algo)
    want, rw, _ = b.render(48, 36, 48, 36, 4, 1, 8, records=True)
    b.close()
    r = compare_records(rg, rw)
    assert r["hash"] == 0 and r["rgb"] == 0 and r["rgb_bit_exact"] == r["n"], r
    np.testing.assert_array_equal(got, want)
    assert not np.array_equal(before, got)


def test_edits_that_change_the_light_list_are_refused(workdir):
    scene, cam = scene_and_camera("all_lights_novol", workdir)
    c = _ctx(scene, cam, "mis")
    before, _, _ = c.render(24, 18, 24, 18, 2, 0, 6)
    arr = ls.scene_arrays(scene)
    floor = {k: arr["meshes"][0][k] for k in ("base_color", "metallic", "roughness", "emission", "transmission", "ior")}
    lit = dict(floor, emission=[1.0, 1.0, 1.0])                    # a non-emitting mesh starts emitting
    ok = dict(floor, base_color=[0.1, 0.1, 0.1])
    for bad in ([{"mesh": 0, "material": lit}], [{"mesh": 99, "material": ok}], [{"light": 42, "desc": arr["lights"][0]}],
                [{"mesh": 0, "material": ok}, {"mesh": 0, "material": lit}]):   # all or none
        assert c.update_scene(bad, check=False) == lucid_capi.LUCID_ERR_INVALID
    after, _, _ = c.render(24, 18, 24, 18, 2, 0, 6)
    np.testing.assert_array_equal(after, before)
    c.close()
    t_scene, t_cam = scene_and_camera("textured", workdir)
    t = _ctx(t_scene, t_cam, "mis")
    tarr = ls.scene_arrays(t_scene, json_rounding=False)
    textured = [i for i, m in enumerate(t_scene["meshes"]) if m.get("material", {}).get("use_nodes")]
    assert textured
    m = {k: tarr["meshes"][textured[0]][k] for k in ("base_color", "metallic", "roughness", "emission", "transmission", "ior")}
    assert t.update_scene([{"mesh": textured[0], "material": m}], check=False) == lucid_capi.LUCID_ERR_INVALID
    t.close()


def _single_call(scene, cam, algo, w, h, spp, depth):
    c = _ctx(scene, cam, algo)
    img, _, _ = c.render(w, h, w, h, spp, 0, depth)
    c.close()
    return img


def test_server_jobs_render_the_version_current_at_submission(workdir):
    """One slot kept busy by a long job; a job queued before an edit and a
    job submitted after it: the first renders the original scene, the
    second the edited one, each bit-identical to a single render call."""
    scene, cam = scene_and_camera("all_lights", workdir)
    edits, edited = _edits_and_edited_scene(scene)
    srv = lucid_capi.Server(0, slots=1)
    sid = srv.add_scene(ls.to_json(scene))
    busy = srv.submit(sid, cam, 320, 240, 256, 8, "volume_mis")
    while srv.state(busy)[0] != lucid_capi.JOB_RUNNING:
        time.sleep(0.001)
    old = srv.submit(sid, cam, 48, 36, 8, 8, "volume_mis")
    srv.update_scene(sid, edits)
    new = srv.submit(sid, cam, 48, 36, 8, 8, "volume_mis")
    for j in (busy, old, new):
        assert srv.wait(j, 120000) == lucid_capi.JOB_DONE
    got_old, got_new, got_busy = srv.result(old), srv.result(new), srv.result(busy)
    srv.close()
    np.testing.assert_array_equal(got_old, _single_call(scene, cam, "volume_mis", 48, 36, 8, 8))
    np.testing.assert_array_equal(got_new, _single_call(edited, cam, "volume_mis", 48, 36, 8, 8))
    np.testing.assert_array_equal(got_busy, _single_call(scene, cam, "volume_mis", 320, 240, 256, 8))


def test_guided_job_is_unbiased_and_leaves_unguided_jobs_unchanged(workdir):
    """A guided job (the guide trained on the job's own samples) beside two
    unguided jobs on two slots: its image mean is within 4 standard errors
    of an FP64 reference of the plain estimator; the unguided jobs equal
    single render calls bit for bit."""
    import lucid_quality as lq
    scene, cam = scene_and_camera("cornell", workdir)
    W, H, SPP = 64, 64, 512
    srv = lucid_capi.Server(0, slots=2)
    sid = srv.add_scene(ls.to_json(scene))
    g = srv.submit(sid, cam, W, H, SPP, 8, "mis", guided=True, guide_seed=3)
    u1 = srv.submit(sid, cam, 48, 48, 16, 8, "mis")
    u2 = srv.submit(sid, cam, 32, 32, 32, 6, "nee", interactive=True)
    for j in (g, u1, u2):
        assert srv.wait(j, 120000) == lucid_capi.JOB_DONE
    gimg, i1, i2 = srv.result(g), srv.result(u1), srv.result(u2)
    srv.close()
    np.testing.assert_array_equal(i1, _single_call(scene, cam, "mis", 48, 48, 16, 8))
    np.testing.assert_array_equal(i2, _single_call(scene, cam, "nee", 32, 32, 32, 6))
    c = _ctx(scene, cam, "mis")
    ref = lq.render_reference(c, W, H, spp=4096, max_depth=8, sample_offset=1 << 20)
    # per-pixel sample variance of the plain estimator for the standard error
    s1 = c.render_f64(W, H, W, H, 256, 1 << 22, 8)[..., :3] / 256
    c.close()
    mean_g = gimg[..., :3].astype(np.float64) / SPP
    lum = lambda x: x @ np.array([0.2126, 0.7152, 0.0722])
    diff = lum(mean_g).mean() - lum(ref).mean()
    # the image mean's standard error from the pixel spread of a 256-spp
    # plain image (the guided estimator's own variance is of the same order)
    se = np.sqrt(np.var(lum(s1) - lum(ref)) * 256 / SPP / (W * H)) + 1e-6
    assert abs(diff) < 4 * se + 2e-3 * abs(lum(ref).mean()), (diff, se)
