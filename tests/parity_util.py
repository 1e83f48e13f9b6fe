"""Helpers shared by the parity tests: render the same scene with the CUDA
tracer (through the C ABI) and with the CPU oracle and compare per-sample
records."""
from __future__ import annotations

import numpy as np

# Per-sample radiance tolerance (relative, with an absolute floor for
# near-zero channels): the target is 1e-4 relative FP32 agreement.
RTOL = 1e-4
ATOL = 1e-6


def scene_and_camera(name: str, workdir: str):
    import lucid_scenes as ls
    if name == "cornell":
        return ls.cornell_box()
    if name == "all_lights":
        return ls.all_lights_scene(workdir=workdir)
    if name == "all_lights_novol":
        return ls.all_lights_scene(workdir=workdir, with_volume=False)
    if name == "two_volumes":
        # a second volume box (a second group of boundary triangles, each
        # group behind its own box test in the closest-hit kernels)
        import os
        sc, cam = ls.all_lights_scene(workdir=workdir)
        sidecar = os.path.join(workdir, "second_volume_grid.f32")
        ls.write_constant_grid(sidecar, (4, 4, 4), 1.0)
        sc["meshes"].append(ls.volume_box_mesh((-2.2, 0.0, -2.0), (-1.0, 1.2, -0.8), 0.8, (0.6, 0.8, 0.9), -0.2,
                                               sidecar, (4, 4, 4)))
        return sc, cam
    if name == "mirror":
        return ls.mirror_point_light_scene()
    if name == "procedural_small":
        return ls.procedural_scene(seed=5, n_spheres=6, levels=2, emissive_levels=1, workdir=workdir, extent=6.0)
    if name == "empty_env":
        # no geometry: every camera ray escapes to the environment
        return ({"meshes": [], "native_lights": [], "environment": {"color": [0.3, 0.4, 0.5], "strength": 1.5}},
                (0.0, 0.0, 3.0, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 45.0))
    if name == "two_small_quads":
        # four triangles, none large against the scene: the whole BVH is one leaf
        m = ls.material((0.7, 0.6, 0.5), 0.0, 0.4)
        meshes = [ls.mesh(*ls.quad((-3, 0, 0), (-2, 0, 0), (-2, 1, 0), (-3, 1, 0)), m),
                  ls.mesh(*ls.quad((2, 0, -4), (3, 0, -4), (3, 1, -4), (2, 1, -4)), ls.material((0.9, 0.9, 0.9), 1.0, 0.2))]
        lights = [{"type": "POINT", "position": [0.0, 2.0, 2.0], "color": [1, 1, 1], "energy": 200.0, "radius": 0.0}]
        return ({"meshes": meshes, "native_lights": lights, "environment": {"color": [0.05, 0.05, 0.08], "strength": 1.0}},
                (0.0, 0.5, 6.0, 0.0, 0.0, -1.0, 0.0, 1.0, 0.0, 60.0))
    if name == "material_preview":
        return ls.material_preview_scene()
    if name == "hard_indirect":
        return ls.hard_indirect_scene()
    if name == "textured":
        return ls.textured_scene()
    raise KeyError(name)


def render_oracle(scene, cam, algo, w, h, spp, depth, offset=0, device_math=True, tile=None):
    import lucid_scenes as ls
    from oracle_ctypes import Oracle
    o = Oracle(device_math=device_math, canonical_ties=True)
    assert o.load_scene_json(ls.to_json(scene))
    o.set_camera(*cam)
    o.set_algorithm(algo)
    tx, ty, tw, th = tile if tile else (0, 0, w, h)
    img, recs, rc = o.render(tw, th, w, h, spp, offset, depth, tile_x=tx, tile_y=ty, records=True)
    assert rc == 0
    return img, recs


def render_gpu(ctx, scene, cam, algo, w, h, spp, depth, offset=0, tile=None):
    import lucid_scenes as ls
    ctx.load_scene_json(ls.to_json(scene))
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    tx, ty, tw, th = tile if tile else (0, 0, w, h)
    img, recs, rc = ctx.render(tw, th, w, h, spp, offset, depth, tile_x=tx, tile_y=ty, records=True)
    return img, recs


def compare_records(gpu, cpu):
    """Returns a dict of mismatch counts; radiance is compared on samples
    whose event hash matches."""
    n = len(cpu)
    prim = (gpu["primary_mesh"] != cpu["primary_mesh"]) | (gpu["primary_tri"] != cpu["primary_tri"])
    hsh = gpu["hash"] != cpu["hash"]
    cnt = (gpu["bounces"] != cpu["bounces"]) | (gpu["nee_tests"] != cpu["nee_tests"]) | \
          (gpu["nee_occluded"] != cpu["nee_occluded"])
    same = ~hsh
    g, c = gpu["rgb"][same], cpu["rgb"][same]
    bad_rgb = ~np.all(np.abs(g - c) <= RTOL * np.abs(c) + ATOL, axis=1) & np.all(np.isfinite(c), axis=1)
    nan_mismatch = np.isnan(g).any(axis=1) != np.isnan(c).any(axis=1)
    exact = np.all(g.view(np.uint32) == c.view(np.uint32), axis=1)
    return {"n": n, "primary": int(prim.sum()), "hash": int(hsh.sum()), "counts": int(cnt.sum()),
            "rgb": int(bad_rgb.sum() + nan_mismatch.sum()), "rgb_bit_exact": int(exact.sum()),
            "max_rel": float(np.max(np.abs(g - c) / (np.abs(c) + 1e-6))) if len(c) else 0.0}
