"""Binary scene upload (lucid_cuda_load_scene_arrays): the array form of a
scene flattens to exactly the device-ready scene its JSON form does (host
digests, no GPU), and renders bit-identically (GPU)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import lucid_capi
import lucid_scenes as ls
from parity_util import scene_and_camera

SCENES = ["cornell", "all_lights", "mirror", "material_preview", "two_small_quads", "empty_env", "procedural_small"]


@pytest.mark.parametrize("name", SCENES)
def test_array_and_json_forms_flatten_identically(name, workdir):
    sc, _ = scene_and_camera(name, workdir)
    assert lucid_capi.scene_digest(json_text=ls.to_json(sc)) == lucid_capi.scene_digest(arrays=ls.scene_arrays(sc))


def test_digest_sees_a_one_ulp_change(workdir):
    sc, _ = scene_and_camera("cornell", workdir)
    arr = ls.scene_arrays(sc)
    d0 = lucid_capi.scene_digest(arrays=arr)
    arr["meshes"][0]["vertices"][4] = np.nextafter(arr["meshes"][0]["vertices"][4], np.float32(np.inf))
    assert lucid_capi.scene_digest(arrays=arr) != d0


def test_malformed_arrays_are_rejected(workdir):
    sc, _ = scene_and_camera("cornell", workdir)
    arr = ls.scene_arrays(sc)
    arr["meshes"][1]["triangles"][0] = 10_000          # index past the vertex array
    with pytest.raises(lucid_capi.LucidError):
        lucid_capi.scene_digest(arrays=arr)
    arr = ls.scene_arrays(sc)
    arr["meshes"][0]["volume_dims"] = (1, 4, 4)        # grid dims below 2
    with pytest.raises(lucid_capi.LucidError):
        lucid_capi.scene_digest(arrays=arr)
    lib = lucid_capi.load_library()
    out = ctypes.c_uint64(0)
    assert lib.lucid_scene_digest(None, 0, None, ctypes.byref(out)) == lucid_capi.LUCID_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("name,algo", [("cornell", "mis"), ("all_lights", "volume_mis"), ("two_small_quads", "nee")])
def test_array_upload_renders_bit_identically(name, algo, workdir):
    sc, cam = scene_and_camera(name, workdir)
    c = lucid_capi.Context(0)
    imgs, stats = [], []
    for form in ("json", "arrays"):
        if form == "json":
            c.load_scene_json(ls.to_json(sc))
        else:
            c.load_scene_arrays(ls.scene_arrays(sc))
        c.set_camera(*cam)
        c.set_algorithm(algo)
        stats.append(c.scene_stats())
        imgs.append(c.render(48, 40, 48, 40, 4, 0, 8)[0].copy())
    c.close()
    assert stats[0] == stats[1]
    assert np.array_equal(imgs[0], imgs[1])


def test_large_json_parsed_in_parallel_matches_the_arrays(workdir):
    """Scenes above 8 MB of JSON are read mesh by mesh on all host threads;
    the result is the scene the array form gives."""
    sc, _ = ls.procedural_scene(seed=4, n_spheres=40, levels=4, emissive_levels=2, workdir=workdir, extent=20.0)
    js = ls.to_json(sc)
    assert len(js) > (8 << 20)
    assert lucid_capi.scene_digest(json_text=js) == lucid_capi.scene_digest(arrays=ls.scene_arrays(sc))


def test_large_json_errors_are_reported(workdir):
    sc, _ = ls.procedural_scene(seed=4, n_spheres=40, levels=4, emissive_levels=2, workdir=workdir, extent=20.0)
    sc["meshes"][5]["triangles"] = np.array(sc["meshes"][5]["triangles"])
    sc["meshes"][5]["triangles"][3, 1] = 10 ** 7                # past the vertex array
    js = ls.to_json(sc)
    with pytest.raises(lucid_capi.LucidError):
        lucid_capi.scene_digest(json_text=js)
    bad = js.replace('"vertices"', '"vertices" x', 1)             # a syntax error inside one mesh
    with pytest.raises(lucid_capi.LucidError):
        lucid_capi.scene_digest(json_text=bad)
