"""GPU parity on the benchmark configurations themselves, against the CPU
oracle, sample by sample (primary hit, path event hash, bounce and shadow
counts, FP32 radiance within 1e-4 relative):

* the Cornell box at its full size: 256x256, 16 samples per pixel in one call,
  `mis`, depth 8;
* the ~1M-triangle procedural scene that bench.py renders (seed 2: 200
  displaced icospheres, ground, emissive spheres, 29 native lights, a volume
  box), `volume_mis`, depth 16, on a stratified crop: the bench's CPU-baseline
  crop (5x4 tiles of 64x33 px spread over the 1920x1080 frame) at 4 samples
  per pixel, and four 16x16 tiles at the full 64 samples per pixel, with a
  non-zero sample offset.

The oracle runs with the shared deterministic math and the canonical
equal-distance tie rule.  A second test runs the oracle in its
reference-literal mode (libm transcendentals, the reference's traversal order
and tie rule, its slab test) and reports how often a sample's event sequence
differs from the GPU's and how far the images are apart.
"""
import numpy as np
import pytest

from parity_util import compare_records

pytestmark = pytest.mark.gpu

C2_W, C2_H, C2_DEPTH, C2_ALGO = 1920, 1080, 16, "volume_mis"


def _c2_tiles():
    nx, ny, tw, th = 5, 4, 64, 33
    tiles = []
    for j in range(ny):
        for i in range(nx):
            tiles.append((int((i + 0.5) * C2_W / nx - tw / 2), int((j + 0.5) * C2_H / ny - th / 2), tw, th))
    return tiles


FULL_SPP_TILES = [(200, 700, 16, 16), (900, 520, 16, 16), (1500, 300, 16, 16), (1700, 980, 16, 16)]


@pytest.fixture(scope="module")
def ctx():
    import lucid_capi
    c = lucid_capi.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def c2_scene(tmp_path_factory):
    import lucid_scenes as ls
    d = str(tmp_path_factory.mktemp("c2"))
    sc, cam = ls.procedural_scene(seed=2, workdir=d)
    assert ls.scene_triangle_count(sc) > 1_000_000
    return ls.to_json(sc), cam


def _oracle(js, cam, algo, device_math=True, canonical_ties=True):
    from oracle_ctypes import Oracle
    o = Oracle(device_math=device_math, canonical_ties=canonical_ties)
    assert o.load_scene_json(js)
    o.set_camera(*cam)
    o.set_algorithm(algo)
    return o


def _gpu_tiles(ctx, js, cam, algo, tiles, full_w, full_h, spp, offset, depth):
    ctx.load_scene_json(js)
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    out = []
    for (tx, ty, tw, th) in tiles:
        img, recs, _ = ctx.render(tw, th, full_w, full_h, spp, offset, depth, tile_x=tx, tile_y=ty, records=True)
        out.append((img, recs))
    return out


def _oracle_tiles(o, tiles, full_w, full_h, spp, offset, depth):
    out = []
    for (tx, ty, tw, th) in tiles:
        img, recs, rc = o.render(tw, th, full_w, full_h, spp, offset, depth, tile_x=tx, tile_y=ty, records=True)
        assert rc == 0
        out.append((img, recs))
    return out


def _assert_exact(gpu, cpu, label):
    total = {"n": 0, "primary": 0, "hash": 0, "counts": 0, "rgb": 0, "rgb_bit_exact": 0}
    for (gi, gr), (ci, cr) in zip(gpu, cpu):
        r = compare_records(gr, cr)
        for k in total:
            total[k] += r[k]
        np.testing.assert_allclose(gi, ci, rtol=1e-4, atol=1e-5, err_msg=label)
    print(label, total)
    assert total["primary"] == 0 and total["hash"] == 0 and total["counts"] == 0 and total["rgb"] == 0, total
    return total


def test_cornell_full_size_parity(ctx):
    """Cornell box, 256x256, 16 spp in one call, mis, depth 8 (1,048,576 samples)."""
    import lucid_scenes as ls
    sc, cam = ls.cornell_box()
    js = ls.to_json(sc)
    g = _gpu_tiles(ctx, js, cam, "mis", [(0, 0, 256, 256)], 256, 256, 16, 0, 8)
    c = _oracle_tiles(_oracle(js, cam, "mis"), [(0, 0, 256, 256)], 256, 256, 16, 0, 8)
    t = _assert_exact(g, c, "cornell 256x256x16")
    assert t["n"] == 256 * 256 * 16


def test_procedural_1m_crop_parity(ctx, c2_scene):
    """The bench scene (1.03M triangles, volume_mis, depth 16): the stratified
    20-tile crop at 4 spp and four tiles at the full 64 spp."""
    js, cam = c2_scene
    o = _oracle(js, cam, C2_ALGO)
    g = _gpu_tiles(ctx, js, cam, C2_ALGO, _c2_tiles(), C2_W, C2_H, 4, 5, C2_DEPTH)
    c = _oracle_tiles(o, _c2_tiles(), C2_W, C2_H, 4, 5, C2_DEPTH)
    t = _assert_exact(g, c, "procedural 1M crop 4 spp")
    assert t["n"] == 20 * 64 * 33 * 4
    g = _gpu_tiles(ctx, js, cam, C2_ALGO, FULL_SPP_TILES, C2_W, C2_H, 64, 64, C2_DEPTH)
    c = _oracle_tiles(o, FULL_SPP_TILES, C2_W, C2_H, 64, 64, C2_DEPTH)
    _assert_exact(g, c, "procedural 1M tiles 64 spp")


def _literal_rate(gpu, cpu):
    n = hsh = prim = 0
    num = den = 0.0
    for (gi, gr), (ci, cr) in zip(gpu, cpu):
        n += len(cr)
        hsh += int((gr["hash"] != cr["hash"]).sum())
        prim += int(((gr["primary_mesh"] != cr["primary_mesh"]) | (gr["primary_tri"] != cr["primary_tri"])).sum())
        num += float(np.abs(gi[..., :3] - ci[..., :3]).sum())
        den += float(np.abs(ci[..., :3]).sum())
    return {"samples": n, "hash_mismatch": hsh, "hash_mismatch_rate": hsh / max(n, 1),
            "primary_mismatch": prim, "image_rel_l1": num / max(den, 1e-30)}


def test_reference_literal_mode_mismatch_rate(ctx, c2_scene):
    """How often the GPU's per-sample event sequence differs from the oracle
    run the way the reference runs (libm sin/cos/exp/log/pow, its slab test,
    its traversal order and equal-distance tie rule), on both benchmark
    configurations.  The differences come from last-bit differences of the
    transcendentals, which change a later RNG-driven decision; the images
    still agree within noise."""
    import lucid_scenes as ls
    sc, cam = ls.cornell_box()
    js = ls.to_json(sc)
    o = _oracle(js, cam, "mis", device_math=False, canonical_ties=False)
    g = _gpu_tiles(ctx, js, cam, "mis", [(0, 0, 256, 256)], 256, 256, 16, 0, 8)
    c = _oracle_tiles(o, [(0, 0, 256, 256)], 256, 256, 16, 0, 8)
    r1 = _literal_rate(g, c)
    print("literal mode, cornell 256x256x16 mis:", r1)
    js2, cam2 = c2_scene
    o = _oracle(js2, cam2, C2_ALGO, device_math=False, canonical_ties=False)
    g = _gpu_tiles(ctx, js2, cam2, C2_ALGO, _c2_tiles(), C2_W, C2_H, 4, 5, C2_DEPTH)
    c = _oracle_tiles(o, _c2_tiles(), C2_W, C2_H, 4, 5, C2_DEPTH)
    r2 = _literal_rate(g, c)
    print("literal mode, procedural 1M crop 4 spp volume_mis:", r2)
    # primary hits differ only where the reference's slab test or tie order
    # picks another triangle at an exactly shared edge
    assert r1["primary_mismatch"] <= 0.01 * r1["samples"] and r2["primary_mismatch"] <= 0.01 * r2["samples"]
    assert r1["hash_mismatch_rate"] < 0.15 and r2["hash_mismatch_rate"] < 0.25
    assert r1["image_rel_l1"] < 0.05


def test_c2_crop_in_a_batch_equals_its_own_renders(c2_scene, tmp_path):
    """The bench scene's stratified crop rendered as tiles inside one batch
    (lucid_cuda_render_batch) beside a Cornell job: the kernels that read
    each path's scene from the batch's scene table give every tile the image
    of its own render call on the 1M-triangle BVH, bit for bit."""
    import lucid_capi
    import lucid_scenes as ls
    js, cam = c2_scene
    c2 = lucid_capi.Context(0)
    c2.load_scene_json(js)
    c2.set_camera(*cam)
    c2.set_algorithm(C2_ALGO)
    cb_scene, cb_cam = ls.cornell_box()
    cb = lucid_capi.Context(0)
    cb.load_scene_json(ls.to_json(cb_scene))
    jobs, want = [], []
    for k, (tx, ty, tw, th) in enumerate(_c2_tiles()[:8]):
        jobs.append({"scene": c2, "camera": cam, "tile_x": tx, "tile_y": ty, "width": tw, "height": th,
                     "full_w": C2_W, "full_h": C2_H, "samples": 4, "sample_offset": 64 * k, "max_depth": C2_DEPTH})
        want.append(c2.render(tw, th, C2_W, C2_H, 4, 64 * k, C2_DEPTH, tile_x=tx, tile_y=ty)[0])
        if k == 3:
            jobs.append({"scene": cb, "camera": cb_cam, "width": 64, "height": 64, "samples": 4,
                         "max_depth": C2_DEPTH})
            cb.set_camera(*cb_cam)
            cb.set_algorithm(C2_ALGO)
            want.append(cb.render(64, 64, 64, 64, 4, 0, C2_DEPTH)[0])
    got, _ = c2.render_batch(jobs, C2_ALGO)
    for k in range(len(jobs)):
        np.testing.assert_array_equal(got[k], want[k], err_msg="job %d" % k)
    c2.close()
    cb.close()
