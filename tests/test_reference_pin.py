"""The oracle pinned to the reference itself.

The Lucid reference's own CPU render path (PyRenderer::render_tile and
render_debug, LucidRenderer/cpp_renderer/include/pybind_renderer.hpp:185-439,
with every integrator, BSDF, light, volume, BVH and RNG header it includes and
src/node_evaluator.cpp) is compiled here from its unmodified sources against a
project-written mp-units API shim (oracle/ref_shim/, `make -C oracle ref`).
The oracle restatement, run the way that build runs (libm transcendentals, the
reference's traversal order and tie rule, and the call-argument draws taken
right to left, the order g++ evaluates them), must give the same image bit for
bit.  The product and the GPU parity tests use the oracle with the draws left
to right (the reference's own toolchain), the shared deterministic math and
the canonical tie rule; the literal-mode mismatch test in
test_gpu_parity_configs.py measures that step.

Runs without a GPU.  Skipped only where neither the built library nor the
reference sources are present.
"""
import os

import numpy as np
import pytest

from golden_cases import GOLDEN_DIR
from make_reference_golden import REF_CASES
from parity_util import scene_and_camera

CASES = [
    ("cornell", "mis", 48, 48, 4, 8),
    ("cornell", "nee", 40, 40, 4, 8),
    ("cornell", "simple", 32, 32, 4, 8),
    ("cornell", "mis", 24, 24, 1, 8),
    ("cornell", "mis", 37, 23, 3, 8),
    ("cornell", "mis", 32, 32, 2, 1),
    ("all_lights_novol", "mis", 48, 36, 4, 8),
    ("all_lights_novol", "nee", 32, 24, 2, 8),
    ("all_lights", "volume_mis", 48, 36, 4, 8),
    ("all_lights", "volume_simple", 32, 24, 2, 8),
    ("mirror", "mis", 32, 32, 4, 6),
    ("procedural_small", "volume_mis", 40, 24, 2, 12),
    ("empty_env", "mis", 16, 16, 2, 4),
    ("two_small_quads", "nee", 32, 24, 2, 6),
    ("material_preview", "mis", 32, 32, 2, 8),
    ("hard_indirect", "mis", 40, 24, 2, 8),
    ("textured", "mis", 48, 36, 4, 8),
    ("textured", "nee", 40, 30, 2, 6),
]


@pytest.fixture(scope="module")
def ref_lib():
    import ref_ctypes
    path = os.path.join(ref_ctypes.REF_DIR, "libref_check.so")
    if os.path.isdir(ref_ctypes.REF_SOURCES):
        ref_ctypes.build()
    if not os.path.exists(path):
        pytest.skip("reference sources absent and the reference library not built")
    return path


def _pair(ref_lib, js, cam, algo):
    import ref_ctypes
    from oracle_ctypes import Oracle
    r = ref_ctypes.ReferenceRenderer(ref_lib)
    assert r.load_scene_json(js)
    r.set_camera(*cam)
    r.set_algorithm(algo)
    o = Oracle(device_math=False, canonical_ties=False, draw_rtl=True)
    assert o.load_scene_json(js)
    o.set_camera(*cam)
    o.set_algorithm(algo)
    return r, o


def _assert_bit_equal(a, b, label):
    same = a.view(np.uint32) == b.view(np.uint32)
    assert same.all(), f"{label}: {int((~same.all(axis=-1)).sum())} pixels differ, max |d| {np.abs(a - b).max()}"


@pytest.mark.parametrize("scene,algo,w,h,spp,depth", CASES)
def test_oracle_reproduces_reference_render_tile(ref_lib, workdir, scene, algo, w, h, spp, depth):
    import lucid_scenes as ls
    sc, cam = scene_and_camera(scene, workdir)
    js = ls.to_json(sc)
    r, o = _pair(ref_lib, js, cam, algo)
    want = r.render(w, h, w, h, spp, 3, depth)
    got, _, rc = o.render(w, h, w, h, spp, 3, depth)
    assert rc == 0
    assert np.isfinite(want).all()
    _assert_bit_equal(got, want, f"{scene}/{algo}")


def test_oracle_reproduces_reference_cornell_full_size(ref_lib):
    """The Cornell configuration at its full size: 256x256, 16 spp, mis, depth 8."""
    import lucid_scenes as ls
    sc, cam = ls.cornell_box()
    r, o = _pair(ref_lib, ls.to_json(sc), cam, "mis")
    want = r.render(256, 256, 256, 256, 16, 0, 8)
    got, _, rc = o.render(256, 256, 256, 256, 16, 0, 8)
    assert rc == 0
    _assert_bit_equal(got, want, "cornell 256x256x16")


def test_oracle_reproduces_reference_tiles_of_a_frame(ref_lib, workdir):
    """Tiles of a larger frame (seeds and camera rays use global pixel
    coordinates), including one that touches the frame's edge."""
    import lucid_scenes as ls
    sc, cam = scene_and_camera("all_lights", workdir)
    r, o = _pair(ref_lib, ls.to_json(sc), cam, "volume_mis")
    for (tx, ty, tw, th) in [(0, 0, 24, 16), (100, 60, 40, 30), (296, 224, 24, 16)]:
        want = r.render(tw, th, 320, 240, 3, 9, 8, tile_x=tx, tile_y=ty)
        got, _, rc = o.render(tw, th, 320, 240, 3, 9, 8, tile_x=tx, tile_y=ty)
        assert rc == 0
        _assert_bit_equal(got, want, f"tile {tx},{ty}")


@pytest.mark.parametrize("scene", ["all_lights", "textured"])
def test_oracle_reproduces_reference_debug_passes(ref_lib, workdir, scene):
    import lucid_scenes as ls
    sc, cam = scene_and_camera(scene, workdir)
    r, o = _pair(ref_lib, ls.to_json(sc), cam, "mis")
    for mode, name in enumerate(["normal", "albedo", "emission"]):
        want = r.render_debug(name, 40, 30)
        got = o.render_debug(mode, 40, 30)
        _assert_bit_equal(got, want, name)


def test_oracle_reproduces_reference_procedural_1m_crop(ref_lib, tmp_path_factory):
    """The ~1M-triangle bench scene (volume_mis, depth 16) on the bench's
    stratified crop: 20 tiles of 64x33 px over the 1920x1080 frame, 4 spp."""
    import lucid_scenes as ls
    d = str(tmp_path_factory.mktemp("c2pin"))
    sc, cam = ls.procedural_scene(seed=2, workdir=d)
    r, o = _pair(ref_lib, ls.to_json(sc), cam, "volume_mis")
    nx, ny, tw, th = 5, 4, 64, 33
    for j in range(ny):
        for i in range(nx):
            tx, ty = int((i + 0.5) * 1920 / nx - tw / 2), int((j + 0.5) * 1080 / ny - th / 2)
            want = r.render(tw, th, 1920, 1080, 4, 5, 16, tile_x=tx, tile_y=ty)
            got, _, rc = o.render(tw, th, 1920, 1080, 4, 5, 16, tile_x=tx, tile_y=ty)
            assert rc == 0
            _assert_bit_equal(got, want, f"tile {tx},{ty}")


@pytest.mark.parametrize("name", list(REF_CASES))
def test_oracle_reproduces_reference_golden_images(workdir, name):
    """Committed images made by the reference itself
    (tests/golden/make_reference_golden.py); needs neither the reference
    sources nor its library."""
    import lucid_scenes as ls
    from oracle_ctypes import Oracle
    scene, algo, w, h, spp, depth, off = REF_CASES[name]
    want = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))["image"]
    sc, cam = scene_and_camera(scene, workdir)
    o = Oracle(device_math=False, canonical_ties=False, draw_rtl=True)
    assert o.load_scene_json(ls.to_json(sc))
    o.set_camera(*cam)
    if algo.startswith("debug:"):
        got = o.render_debug(["normal", "albedo", "emission"].index(algo.split(":", 1)[1]), w, h)
    else:
        o.set_algorithm(algo)
        got, _, rc = o.render(w, h, w, h, spp, off, depth)
        assert rc == 0
    _assert_bit_equal(got, want, name)


DIAG_CASES = [
    ("cornell", "mis", 24, 24, 4, 8, 2),
    ("cornell", "nee", 16, 16, 3, 8, 1),
    ("cornell", "simple", 16, 16, 2, 6, 2),
    ("all_lights_novol", "mis", 24, 16, 2, 8, 2),
    ("mirror", "mis", 16, 16, 4, 6, 1),
]


@pytest.mark.parametrize("scene,algo,w,h,spp,depth,sf", DIAG_CASES)
def test_oracle_reproduces_reference_diagnostic_render(ref_lib, workdir, scene, algo, w, h, spp, depth, sf):
    """render_tile with diagnostics enabled (the reference's diagnostic
    integrators, path_tracer.hpp:880-1514, recording into a fresh
    DiagnosticFilm per call, pybind_renderer.hpp:205-316): the image, the
    global stats and every pixel's get_pixel_diagnostic (sample / group /
    outlier counts, variance, mean, and each group's object ids, counts,
    mean and variance, depth, coarse type, strategy, vertex positions and
    normals) equal the oracle's restatement.

    The reference parallelises the pixels of each 8x8 micro-tile over
    OpenMP threads, so with a subsample factor above 1 several threads
    update one film cell at once (a data race: samples counted, groups
    lost).  It runs single-threaded here, in the loop order the oracle and
    the CUDA film replay follow."""
    import lucid_scenes as ls
    sc, cam = scene_and_camera(scene, workdir)
    r, o = _pair(ref_lib, ls.to_json(sc), cam, algo)
    r.enable_diagnostics(subsample=sf)
    r.set_threads(1)
    try:
        want_img = r.render(w, h, w, h, spp, 2, depth)
    finally:
        r.set_threads(0)
    want = r.diag_report(w, h, top_n=8)
    got_img, rc = o.render_diag(w, h, w, h, spp, 2, depth, subsample=sf)
    assert rc == 0
    _assert_bit_equal(got_img, want_img, f"{scene}/{algo} diagnostic image")
    assert o.diag_stats()[:4] == want["stats"]
    f32 = np.float32
    n_groups = 0
    for y in range(h):
        for x in range(w):
            wp = want["pixels"][y * w + x]
            info, groups = o.diag_pixel(x, y)
            assert bool(info["valid"]) == wp["valid"]
            if not wp["valid"]:
                continue
            assert (int(info["sample_count"]), int(info["group_count"]), int(info["outlier_count"])) == \
                (wp["samples"], wp["groups"], wp["outliers"]), (x, y)
            assert f32(info["variance"]) == f32(wp["variance"])
            assert [f32(v) for v in info["mean_rgb"]] == [f32(v) for v in wp["mean_rgb"]]
            assert len(groups) == len(wp["top"])
            for g, wg in zip(groups, wp["top"]):
                d = int(g["depth"])
                assert d == wg["depth"] and int(g["count"]) == wg["count"]
                assert [int(v) for v in g["object_ids"][:d]] == wg["object_ids"]
                assert int(g["coarse_type"]) == wg["coarse_type"]
                assert ["BSDF", "NEE", "MIS_BSDF", "MIS_NEE"][int(g["strategy"])] == wg["strategy"]
                assert [f32(v) for v in g["mean_rgb"]] == [f32(v) for v in wg["mean_rgb"]]
                assert [f32(v) for v in g["variance_rgb"]] == [f32(v) for v in wg["variance_rgb"]]
                assert f32(g["mean_luminance"]) == f32(wg["mean_luminance"])
                assert g["positions"][:d].astype(np.float32).tolist() == \
                    np.asarray(wg["positions"][1:], np.float32).tolist()
                assert g["normals"][:d].astype(np.float32).tolist() == np.asarray(wg["normals"], np.float32).tolist()
                n_groups += 1
    assert n_groups > 0
    r.disable_diagnostics()
