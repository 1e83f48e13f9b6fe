"""Path diagnostics (DiagnosticFilm): the diagnostic integrators and the
per-pixel path-group statistics.

CPU tests pin the oracle's restatement (diagnostic radiance equals the
normal integrator for MIS and NEE, group hashes and coarse types follow
path_types.hpp:321-372, top groups are sorted) and the Python surface
without a GPU.  GPU tests compare the CUDA diagnostic render and its film,
cell by cell and group by group, with the oracle's."""
from __future__ import annotations

import numpy as np
import pytest

import lucid_scenes as ls
from parity_util import scene_and_camera

FNV_OFFSET = 14695981039346656037
FNV_PRIME = 1099511628211
MASK = (1 << 64) - 1


def path_hash(depth, object_ids, bsdf, flags):
    """PathTrace::hash (path_types.hpp:321-343); the material id is 0 for a
    surface vertex and -1 for the final Emission vertex."""
    h = FNV_OFFSET
    h = ((h ^ depth) * FNV_PRIME) & MASK
    for i in range(depth):
        material = -1 if bsdf[i] == 4 else 0
        for v in (int(object_ids[i]) & MASK, material & MASK, int(bsdf[i]), int(flags[i])):
            h = ((h ^ v) * FNV_PRIME) & MASK
    return h


def coarse_type(depth, flags):
    t = 0
    for i in range(depth):
        if flags[i] & 2:
            t |= 1
        if flags[i] & 1:
            t |= 2
    if depth > 2:
        t |= 4
    return t


def floor_wall_octahedron_scene():
    """A floor, a back wall and a small glossy octahedron under a point light,
    viewed from the front (z up): the shape of the reference's PyRenderer
    diagnostics test scene (test_pyrenderer_diagnostics.cpp:280-333)."""
    oct_v = np.array([[0, 0, 0.5], [0.3, 0, 0.35], [-0.3, 0, 0.35], [0, 0.3, 0.35], [0, -0.3, 0.35], [0, 0, 0.2]])
    oct_t = np.array([[0, 1, 3], [0, 3, 2], [0, 2, 4], [0, 4, 1], [5, 1, 4], [5, 4, 2], [5, 2, 3], [5, 3, 1]])
    meshes = [ls.mesh(*ls.quad((-2, -2, 0), (2, -2, 0), (2, 2, 0), (-2, 2, 0)), ls.material((0.8, 0.8, 0.8), 0.0, 0.9)),
              ls.mesh(*ls.quad((-2, 2, 0), (2, 2, 0), (2, 2, 3), (-2, 2, 3)), ls.material((0.7, 0.7, 0.7), 0.0, 0.9)),
              ls.mesh(oct_v, oct_t, ls.material((0.3, 0.6, 0.9), 0.7, 0.4))]
    lights = [{"type": "POINT", "position": [0.0, -1.0, 2.5], "color": [1, 1, 1], "energy": 50.0, "radius": 0.0}]
    scene = {"meshes": meshes, "native_lights": lights, "environment": {"color": [0.0, 0.0, 0.0], "strength": 1.0}}
    camera = (0.0, -2.5, 1.5, 0.0, 0.5, -0.2, 0.0, 0.0, 1.0, 60.0)
    return scene, camera


def oracle_for(scene, cam, algo):
    from oracle_ctypes import Oracle
    o = Oracle(device_math=True, canonical_ties=True)
    assert o.load_scene_json(ls.to_json(scene))
    o.set_camera(*cam)
    o.set_algorithm(algo)
    return o


# ---------------------------------------------------------------- CPU: oracle
@pytest.mark.parametrize("name,algo", [("cornell", "mis"), ("cornell", "nee"), ("mirror", "mis"),
                                       ("all_lights_novol", "mis"), ("octahedron", "mis")])
def test_oracle_diagnostic_render_matches_normal(oracle_lib, workdir, name, algo):
    """DiagnosticRenderMatchesNormal (test_pyrenderer_diagnostics.cpp:353-369):
    with no volumes in the scene the diagnostic integrator returns the normal
    integrator's radiance."""
    scene, cam = floor_wall_octahedron_scene() if name == "octahedron" else scene_and_camera(name, workdir)
    o = oracle_for(scene, cam, algo)
    img_n, _, rc = o.render(12, 10, samples=3, sample_offset=42, max_depth=6)
    assert rc == 0
    img_d, rc = o.render_diag(12, 10, samples=3, sample_offset=42, max_depth=6, subsample=2)
    assert rc == 0
    np.testing.assert_array_equal(img_n, img_d)
    st = o.diag_stats()
    assert st[0] > 0 and st[0] == st[4] and st[1] > 0


def test_oracle_exporter_restatement(oracle_lib, workdir):
    """The oracle's DiagnosticExporter: the binary blob's cells are the
    film's cells; at subsample 2 the coarse aggregation reads every cell once,
    so its counts sum to the samples recorded; at subsample 4 it reads only the
    cells at (2 sx, 2 sy) (the exporter's fixed factor)."""
    scene, cam = scene_and_camera("all_lights_novol", workdir)
    for sf in (2, 4):
        o = oracle_for(scene, cam, "mis")
        w, h = 16, 12
        _, rc = o.render_diag(w, h, samples=8, max_depth=6, subsample=sf)
        assert rc == 0
        hdr, cells = parse_pvar(o.diag_export_binary())
        assert hdr == (1, w, h, w // sf, h // sf, sf, 16, 4)
        k = 0
        for y in range(0, h // sf * sf, sf):
            for x in range(0, w // sf * sf, sf):
                info, _ = o.diag_pixel(x, y)
                assert cells["gc"][k] == info["group_count"] and cells["ts"][k] == info["sample_count"]
                np.testing.assert_array_equal(cells["mean"][k], info["mean_rgb"])
                assert cells["var"][k] == info["variance"]
                k += 1
        coarse = o.diag_coarse()
        assert [c[1] for c in coarse][:2] == ["Direct-NoDelta-BSDF", "Direct-NoDelta-NEE"]
        want = 0
        for sy in range(h // sf):
            for sx in range(w // sf):
                cx, cy = 2 * sx // sf, 2 * sy // sf          # the cell that film position (2 sx, 2 sy) falls in
                if cx < w // sf and cy < h // sf:
                    want += int(o.diag_pixel(cx * sf, cy * sf)[0]["sample_count"])
        assert sum(c[2] for c in coarse) == want
        assert set(o.diag_suggestion_kinds()) <= {0, 1, 2, 3}


def test_oracle_film_invariants(oracle_lib, workdir):
    scene, cam = scene_and_camera("all_lights_novol", workdir)
    o = oracle_for(scene, cam, "mis")
    w, h, sf = 16, 12, 2
    _, rc = o.render_diag(w, h, samples=8, max_depth=6, subsample=sf)
    assert rc == 0
    total, active, groups_total, overflow, recorded = o.diag_stats()
    seen_samples = seen_groups = 0
    light_types = set()
    for y in range(0, h, sf):
        for x in range(0, w, sf):
            info, groups = o.diag_pixel(x, y)
            assert info["valid"] == 1
            seen_samples += int(info["sample_count"])
            seen_groups += int(info["group_count"])
            assert len(groups) == info["group_count"] <= 16
            var = groups["total_variance"]
            assert np.all(var[:-1] >= var[1:])          # sorted by variance, descending
            for g in groups:
                d = int(g["depth"])
                assert 1 <= d <= 16
                assert int(g["hash"]) == path_hash(d, g["object_ids"], g["bsdf"], g["flags"])
                assert int(g["coarse_type"]) == coarse_type(d, g["flags"])
                assert g["bsdf"][d - 1] == 4                # ends at an Emission vertex
                light_types.add(int(g["light_type"]))
                assert g["count"] >= 1
            _, by_mean = o.diag_pixel(x, y, sort_by_mean=True)
            ml = by_mean["mean_luminance"]
            assert np.all(ml[:-1] >= ml[1:])
    assert seen_samples == total == recorded
    assert seen_groups == groups_total and active == (w // sf) * (h // sf)
    assert overflow >= 0
    assert {1, 2, 5} <= light_types                          # point, area, environment
    top, xy = o.diag_top_groups(8)
    assert 0 < len(top) <= 8 and np.all(top["count"] >= 2)
    assert np.all(top["total_variance"][:-1] >= top["total_variance"][1:])
    for g, (x, y) in zip(top, xy):
        _, cell = o.diag_pixel(int(x), int(y))
        assert int(g["hash"]) in set(int(c["hash"]) for c in cell)


def test_python_surface_without_gpu():
    import lucidrenderer as lr
    c = lr.PathRecordingConfig.minimal()
    assert (c.subsample_factor, c.max_groups_per_pixel, c.max_outliers_per_pixel, c.max_depth) == (4, 8, 2, 8)
    s = lr.PathRecordingConfig.standard()
    assert (s.subsample_factor, s.max_groups_per_pixel) == (2, 16)
    d = lr.PathRecordingConfig.detailed()
    assert (d.subsample_factor, d.max_groups_per_pixel, d.max_outliers_per_pixel) == (1, 32, 8)
    assert d.estimate_memory_bytes(1920, 1080) > s.estimate_memory_bytes(1920, 1080) > c.estimate_memory_bytes(1920, 1080)
    r = lr.Renderer()
    assert hasattr(lr, "DiagnosticExporter") and hasattr(lr, "ExportedCoarseStats")
    assert not r.is_diagnostics_enabled()
    r.enable_diagnostics(c)
    assert r.is_diagnostics_enabled()
    assert not r.get_pixel_diagnostic(0, 0).valid
    st = r.get_diagnostic_stats()
    assert st.total_samples == 0 and st.active_pixels == 0
    assert r.get_diagnostic_variance_map().size == 0
    assert r.export_diagnostic_json() == "{}"
    assert r.get_top_variance_groups(5) == []
    r.clear_diagnostics()
    r.disable_diagnostics()
    assert not r.is_diagnostics_enabled()
    bad = lr.PathRecordingConfig()
    bad.subsample_factor = 0
    with pytest.raises(ValueError):
        r.enable_diagnostics(bad)


# ---------------------------------------------------------------- GPU: parity with the oracle
@pytest.fixture(scope="module")
def gpu_ctx():
    import lucid_capi
    c = lucid_capi.Context(0)
    yield c
    c.close()


def _gpu_diag(ctx, scene, cam, algo, w, h, spp, depth, offset, sf, record_capacity=0):
    ctx.load_scene_json(ls.to_json(scene))
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    ctx.diag_enable(subsample=sf, record_capacity=record_capacity)
    img, _, rc = ctx.render(w, h, w, h, spp, offset, depth)
    assert rc == 0
    return img


def _compare_films(ctx, o, w, h, sf):
    assert ctx.diag_stats() == o.diag_stats()
    for y in range(0, h, sf):
        for x in range(0, w, sf):
            for by_mean in (False, True):
                gi, gg = ctx.diag_pixel(x, y, sort_by_mean=by_mean)
                oi, og = o.diag_pixel(x, y, sort_by_mean=by_mean)
                for f in ("valid", "sample_count", "group_count", "outlier_count", "overflow_count"):
                    assert gi[f] == oi[f], (x, y, f)
                np.testing.assert_allclose(gi["variance"], oi["variance"], rtol=1e-4, atol=1e-7)
                np.testing.assert_allclose(gi["mean_rgb"], oi["mean_rgb"], rtol=1e-4, atol=1e-7)
                assert len(gg) == len(og)
                for a, b in zip(gg, og):
                    for f in ("hash", "count", "depth", "coarse_type", "light_type", "strategy"):
                        assert a[f] == b[f], (x, y, f)
                    d = int(a["depth"])
                    for f in ("object_ids", "bsdf", "flags"):
                        np.testing.assert_array_equal(a[f][:d], b[f][:d])
                    for f in ("mean_rgb", "variance_rgb", "positions", "normals"):
                        np.testing.assert_allclose(a[f], b[f], rtol=1e-4, atol=1e-6)
    for by_mean in (False, True):
        tg, txy = ctx.diag_top_groups(10, by_mean)
        to, oxy = o.diag_top_groups(10, by_mean)
        np.testing.assert_array_equal(tg["hash"], to["hash"])
        np.testing.assert_array_equal(txy, oxy)
    np.testing.assert_allclose(ctx.diag_variance_map(w, h).reshape(h, w)[::sf, ::sf],
                               np.array([[o.diag_pixel(x, y)[0]["variance"] for x in range(0, w, sf)]
                                         for y in range(0, h, sf)]), rtol=1e-4, atol=1e-7)


def parse_pvar(blob: bytes):
    """DiagnosticFilm::export_binary layout (diagnostic_film.hpp:243-299):
    'PVAR', version, width, height, sampled width, sampled height (uint32),
    subsample, max groups, max outliers, 0 (uint8), then per cell group count
    (uint16), samples (uint32), mean rgb, total variance (float32)."""
    import struct
    assert blob[:4] == b"PVAR"
    version, w, h, sw, sh = struct.unpack_from("<5I", blob, 4)
    sf, mg, mo, pad = struct.unpack_from("<4B", blob, 24)
    cells = np.frombuffer(blob, np.dtype([("gc", "<u2"), ("ts", "<u4"), ("mean", "<f4", 3), ("var", "<f4")]),
                          offset=28)
    assert len(blob) == 28 + 22 * sw * sh and pad == 0
    return (version, w, h, sw, sh, sf, mg, mo), cells


def _compare_exports(ctx, o, w, h, sf):
    hdr, cells = parse_pvar(ctx.diag_export_binary())
    ohdr, ocells = parse_pvar(o.diag_export_binary())
    assert hdr == ohdr == (1, w, h, w // sf, h // sf, sf, 16, 4)
    np.testing.assert_array_equal(cells["gc"], ocells["gc"])
    np.testing.assert_array_equal(cells["ts"], ocells["ts"])
    np.testing.assert_allclose(cells["mean"], ocells["mean"], rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(cells["var"], ocells["var"], rtol=1e-4, atol=1e-7)
    for a, b in zip(ctx.diag_coarse_stats(), o.diag_coarse()):
        assert a[:3] == b[:3]
        np.testing.assert_allclose(np.array(a[3:5]), np.array(b[3:5]), rtol=1e-4, atol=1e-7)
        np.testing.assert_allclose(np.array(a[5] + a[6]), np.array(b[5] + b[6]), rtol=1e-4, atol=1e-7)
    kinds = {"High variance detected in glossy reflections": 0,
             "Significant variance from indirect illumination": 1,
             "High variance in diffuse lighting": 2, "Many path types exceeded tracking capacity": 3}
    assert [kinds[s[2]] for s in ctx.diag_suggestions()] == o.diag_suggestion_kinds()
    st = ctx.diag_stats()
    assert ctx.diag_metadata_json() == (
        f'{{\n  "width": {w},\n  "height": {h},\n  "sampled_width": {w // sf},\n  "sampled_height": {h // sf},\n'
        f'  "subsample_factor": {sf},\n  "max_groups": 16,\n  "max_outliers": 4,\n  "total_samples": {st[4]}\n}}\n')


DIAG_CASES = [("cornell", "mis", 16, 16, 16), ("cornell", "nee", 16, 16, 8), ("cornell", "simple", 16, 16, 8),
              ("mirror", "mis", 16, 12, 8), ("all_lights_novol", "mis", 24, 16, 8),
              ("procedural_small", "nee", 16, 16, 4), ("octahedron", "mis", 16, 16, 8)]


@pytest.mark.gpu
@pytest.mark.parametrize("name,algo,w,h,spp", DIAG_CASES)
def test_gpu_diagnostics_match_oracle(gpu_ctx, workdir, name, algo, w, h, spp):
    scene, cam = floor_wall_octahedron_scene() if name == "octahedron" else scene_and_camera(name, workdir)
    sf, depth, offset = 2, 8, 3
    img = _gpu_diag(gpu_ctx, scene, cam, algo, w, h, spp, depth, offset, sf)
    o = oracle_for(scene, cam, algo)
    oimg, rc = o.render_diag(w, h, samples=spp, sample_offset=offset, max_depth=depth, subsample=sf)
    assert rc == 0
    np.testing.assert_allclose(img, oimg, rtol=1e-4, atol=1e-6)
    _compare_films(gpu_ctx, o, w, h, sf)
    _compare_exports(gpu_ctx, o, w, h, sf)
    gpu_ctx.diag_disable()


@pytest.mark.gpu
def test_gpu_diagnostics_bands_waves_and_regrow(gpu_ctx, workdir):
    """Small waves (several 8-row bands, several sample waves per band) and a
    64-record buffer that must grow: the film is the same as the oracle's."""
    scene, cam = scene_and_camera("cornell", workdir)
    w, h, spp, sf = 20, 28, 12, 1
    gpu_ctx.set_wave_capacity(256)
    try:
        img = _gpu_diag(gpu_ctx, scene, cam, "mis", w, h, spp, 6, 0, sf, record_capacity=64)
    finally:
        gpu_ctx.set_wave_capacity(0)
    o = oracle_for(scene, cam, "mis")
    oimg, rc = o.render_diag(w, h, samples=spp, max_depth=6, subsample=sf)
    assert rc == 0
    np.testing.assert_allclose(img, oimg, rtol=1e-4, atol=1e-6)
    _compare_films(gpu_ctx, o, w, h, sf)
    _compare_exports(gpu_ctx, o, w, h, sf)
    gpu_ctx.diag_disable()


@pytest.mark.gpu
def test_gpu_pyrenderer_diagnostics_workflow():
    """The reference's PyRenderer diagnostics tests (test_pyrenderer_diagnostics.cpp:
    339-475) through the lucidrenderer module."""
    import lucidrenderer as lr
    scene, cam = floor_wall_octahedron_scene()
    r = lr.Renderer()
    assert r.load_scene_json(ls.to_json(scene))
    r.set_camera(*cam)
    r.set_algorithm("mis")
    r.enable_diagnostics(lr.PathRecordingConfig.minimal())
    p1 = np.array(r.render_tile(0, 0, 4, 4, 4, 4, 1, 42, 4))
    r.disable_diagnostics()
    p2 = np.array(r.render_tile(0, 0, 4, 4, 4, 4, 1, 42, 4))
    np.testing.assert_array_equal(p1, p2)

    r.enable_diagnostics(lr.PathRecordingConfig.minimal())
    r.render_tile(0, 0, 8, 8, 8, 8, 16, 0, 4)
    st = r.get_diagnostic_stats()
    assert st.total_samples > 0 and st.active_pixels > 0
    vm = r.get_diagnostic_variance_map()
    assert vm.size == 64 and np.all(vm >= 0)
    js = r.export_diagnostic_json()
    for k in ("width", "height", "total_samples", "subsample_factor"):
        assert k in js
    r.clear_diagnostics()
    assert r.get_diagnostic_stats().total_samples == 0
    r.render_tile(0, 0, 8, 8, 8, 8, 4, 0, 4)
    assert r.get_diagnostic_stats().total_samples > 0

    r.enable_diagnostics(lr.PathRecordingConfig.standard())
    r.render_tile(0, 0, 16, 16, 16, 16, 8, 0, 4)
    groups = r.get_top_variance_groups(5)
    assert 0 < len(groups) <= 5
    assert all(g.sample_count >= 2 for g in groups)
    ex = lr.DiagnosticExporter(r)                       # diagnostic_export.hpp:78-220
    assert ex.get_global_stats().total_samples == r.get_diagnostic_stats().total_samples
    assert [g.signature for g in ex.get_top_variance_groups(5)] == [g.signature for g in groups]
    means = [g.mean_luminance for g in ex.get_top_mean_groups(5)]
    assert means == sorted(means, reverse=True)
    coarse = ex.get_coarse_stats()
    assert [c.type_id for c in coarse] == list(range(8)) and coarse[0].name == "Direct-NoDelta-BSDF"
    blob = ex.export_binary()
    assert blob[:4] == b"PVAR" and len(blob) == 28 + 22 * 8 * 8
    assert '"subsample_factor": 2' in ex.export_metadata_json()
    assert all(s.severity in ("info", "warning", "critical") for s in ex.generate_suggestions())
    info = r.get_pixel_diagnostic(8, 8)
    assert info.valid and info.sample_count > 0 and len(info.top_groups) == info.group_count
    r.set_object_names(["Floor", "BackWall", "Sphere"])
    for g in info.top_groups:
        assert len(g.positions) == g.depth + 1 and len(g.normals) == g.depth
        assert g.positions[0] == pytest.approx(list(cam[:3]))
        assert g.signature_heckbert.endswith(" DSE") and g.strategy_name in ("MIS_BSDF", "MIS_NEE")
        assert g.object_path.endswith("→ Camera")
    by_mean = r.get_pixel_diagnostic(8, 8, "mean").top_groups
    assert [g.mean_luminance for g in by_mean] == sorted([g.mean_luminance for g in by_mean], reverse=True)

    for algo in ("simple", "nee", "mis"):
        r.set_algorithm(algo)
        r.enable_diagnostics(lr.PathRecordingConfig.minimal())
        r.render_tile(0, 0, 4, 4, 4, 4, 2, 0, 4)
        assert r.get_diagnostic_stats().total_samples > 0, algo
        r.clear_diagnostics()
