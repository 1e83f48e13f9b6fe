"""GPU parity: the CUDA wavefront tracer against the CPU oracle.

For every (pixel, sample) the two sides must agree on the primary hit
(mesh, triangle), on the path's event hash (every hit primitive, native
light hit, scatter decision and shadow-ray outcome along the path), on the
bounce / shadow-test counts, and on the FP32 radiance within 1e-4 relative.
The oracle runs with the shared deterministic math and the canonical
equal-distance tie rule (see oracle/lucid_oracle.hpp).
"""
import numpy as np
import pytest

from parity_util import compare_records, render_gpu, render_oracle, scene_and_camera

pytestmark = pytest.mark.gpu

CASES = [
    ("cornell", "mis", 48, 48, 4, 8),
    ("cornell", "nee", 40, 40, 4, 8),
    ("cornell", "simple", 32, 32, 4, 8),
    ("cornell", "mis", 24, 24, 1, 8),          # one sample per call: no jitter draws
    ("all_lights_novol", "mis", 48, 36, 4, 8),
    ("all_lights_novol", "nee", 32, 24, 2, 8),
    ("all_lights", "volume_mis", 48, 36, 4, 8),
    ("all_lights", "volume_simple", 32, 24, 2, 8),
    ("two_volumes", "volume_mis", 40, 30, 2, 8),   # two boundary meshes (two culling groups)
    ("mirror", "mis", 32, 32, 4, 6),
    ("procedural_small", "volume_mis", 40, 24, 2, 12),
    ("cornell", "mis", 37, 23, 3, 8),           # ragged frame: no multiple of the warp or block size
    ("cornell", "mis", 32, 32, 2, 1),           # camera rays only
    ("empty_env", "mis", 16, 16, 2, 4),         # no geometry
    ("two_small_quads", "nee", 32, 24, 2, 6),   # single-leaf BVH
    ("material_preview", "mis", 32, 32, 2, 8),
    ("hard_indirect", "mis", 40, 24, 2, 8),
    ("textured", "mis", 48, 36, 4, 8),          # node-graph materials with UV checker textures
    ("textured", "nee", 40, 30, 2, 6),
]


@pytest.fixture(scope="module")
def ctx():
    import lucid_capi
    c = lucid_capi.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("scene,algo,w,h,spp,depth", CASES)
def test_per_sample_parity(ctx, workdir, scene, algo, w, h, spp, depth):
    sc, cam = scene_and_camera(scene, workdir)
    gimg, grec = render_gpu(ctx, sc, cam, algo, w, h, spp, depth, offset=3)
    cimg, crec = render_oracle(sc, cam, algo, w, h, spp, depth, offset=3)
    r = compare_records(grec, crec)
    print(scene, algo, r)
    assert r["primary"] == 0, r
    assert r["hash"] == 0, r
    assert r["counts"] == 0, r
    assert r["rgb"] == 0, r
    np.testing.assert_allclose(gimg, cimg, rtol=1e-4, atol=1e-5)


def test_tile_equals_full_frame(ctx, workdir):
    """Rendering a tile gives the same pixels as the matching part of the full
    frame (seeds use global pixel coordinates)."""
    sc, cam = scene_and_camera("cornell", workdir)
    full, _ = render_gpu(ctx, sc, cam, "mis", 64, 48, 2, 8)
    tile, _ = render_gpu(ctx, sc, cam, "mis", 64, 48, 2, 8, tile=(16, 8, 24, 20))
    # full is Y-flipped over 48 rows, tile over 20 rows
    full_unflip = full[::-1]
    tile_unflip = tile[::-1]
    assert np.array_equal(full_unflip[8:28, 16:40], tile_unflip)


@pytest.mark.parametrize("scene", ["all_lights", "textured"])
def test_debug_passes_match_oracle(ctx, workdir, scene):
    import lucid_scenes as ls
    from oracle_ctypes import Oracle
    sc, cam = scene_and_camera(scene, workdir)
    ctx.load_scene_json(ls.to_json(sc))
    ctx.set_camera(*cam)
    o = Oracle()
    assert o.load_scene_json(ls.to_json(sc))
    o.set_camera(*cam)
    for mode, name in enumerate(["normal", "albedo", "emission"]):
        g = ctx.render_debug(name, 40, 30)
        c = o.render_debug(mode, 40, 30)
        assert np.array_equal(g, c), name


@pytest.mark.parametrize("name", ["cornell_mis", "cornell_nee", "all_lights_volume_mis", "mirror_mis"])
def test_against_golden_fixtures(ctx, workdir, name):
    """The CUDA tracer reproduces the committed oracle fixtures
    (tests/golden/make_golden.py) without running the oracle."""
    from golden_cases import GOLDEN, load_golden
    scene, algo, w, h, spp, depth, off = GOLDEN[name]
    sc, cam = scene_and_camera(scene, workdir)
    gimg, grec = render_gpu(ctx, sc, cam, algo, w, h, spp, depth, offset=off)
    fimg, frec = load_golden(name)
    r = compare_records(grec, frec)
    assert r["primary"] == 0 and r["hash"] == 0 and r["counts"] == 0 and r["rgb"] == 0, r
    np.testing.assert_allclose(gimg, fimg, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("scene,algo", [("cornell", "mis"), ("all_lights", "volume_mis"), ("procedural_small", "nee")])
def test_launch_profiles_give_identical_samples(ctx, workdir, scene, algo):
    """The launch profiles change only the kernels' resident CTAs per SM (and
    so their register caps): every sample stays bit-identical."""
    sc, cam = scene_and_camera(scene, workdir)
    out = []
    for prof in (0, 1):
        ctx.set_launch_profile(prof)
        out.append(render_gpu(ctx, sc, cam, algo, 40, 30, 4, 8, offset=2))
    ctx.set_launch_profile(0)
    (i0, r0), (i1, r1) = out
    assert np.array_equal(r0["hash"], r1["hash"])
    assert np.array_equal(i0.view(np.uint32), i1.view(np.uint32))
