"""The reference module's standalone diagnostics classes (DiagnosticFilm,
DiagnosticPathTracer, DiagnosticExporter(film), PathTrace,
PathDiagnosticRecorder, BsdfType, LightSourceType;
LucidRenderer/cpp_renderer/src/pybind_module.cpp:433-539) on the lucidrenderer
module, run without a GPU:

* the add-on's own caller, LucidRenderer/diagnostics.py (DiagnosticsManager),
  loaded unchanged from the reference where it is present, works on this
  module: the workflows of LucidRenderer/tests/test_diagnostics_python.py
  (full workflow, binary export, clear) re-expressed;
* a seeded stream of paths fed to the reference's own DiagnosticFilm through
  its own PathDiagnosticRecorder (built here, oracle/_ref) and to this module's
  gives the same film: every cell's sample / group / overflow / outlier counts
  and group hashes, the global stats, the exporter's top groups, coarse
  stats, suggestions, metadata JSON and binary blob.
"""
import importlib.util
import os

import numpy as np
import pytest

REF_ADDON = "/root/reference/LucidRenderer/diagnostics.py"


@pytest.fixture(scope="module")
def lr():
    import lucidrenderer
    return lucidrenderer


def test_surface_exists(lr):
    for name in ("DiagnosticFilm", "DiagnosticPathTracer", "DiagnosticExporter", "PathTrace",
                 "PathDiagnosticRecorder", "BsdfType", "LightSourceType", "PathRecordingConfig"):
        assert hasattr(lr, name), name
    assert int(lr.BsdfType.Glass) == 3 and int(lr.LightSourceType.Emissive) == 6


def test_recorder_and_trace(lr):
    rec = lr.PathDiagnosticRecorder()
    rec.begin_path()
    rec.record_vertex(0, 0, lr.BsdfType.Diffuse, False, True)
    rec.record_vertex(3, 1, lr.BsdfType.Mirror, True, False)
    rec.record_light_hit(2, lr.LightSourceType.Spot)
    assert rec.current_depth() == 3
    t = rec.end_path(0.5, 0.25, 2.0)
    assert t.depth == 3
    assert list(t.get_contribution()) == [0.5, 0.25, 2.0]
    rec.begin_path()
    assert rec.current_depth() == 0
    assert lr.PathTrace().depth == 0


def test_film_and_tracer(lr):
    cfg = lr.PathRecordingConfig.standard()
    film = lr.DiagnosticFilm(64, 48, cfg)
    assert (film.width(), film.height(), film.sampled_width(), film.sampled_height()) == (64, 48, 32, 24)
    rec = lr.PathDiagnosticRecorder()
    rec.begin_path()
    rec.record_vertex(1, 0, lr.BsdfType.Glossy, False, False)
    rec.record_environment_hit()
    film.record_path(10, 10, rec.end_path_lum(0.75))
    film.record_path(64, 0, rec.end_path_lum(0.75))      # outside the film: ignored
    assert film.total_paths_recorded() == 1
    st = film.global_stats()
    assert (st.total_samples, st.active_pixels, st.total_groups) == (1, 1, 1)
    assert '"total_samples": 1' in film.metadata_json()
    film.clear()
    assert film.total_paths_recorded() == 0 and film.global_stats().total_samples == 0
    tracer = lr.DiagnosticPathTracer(32, 32, lr.PathRecordingConfig.minimal())
    assert tracer.is_enabled()
    tracer.set_enabled(False)
    assert not tracer.is_enabled()
    f = tracer.film()
    assert f.sampled_width() == 8
    ex = lr.DiagnosticExporter(f)
    assert ex.get_global_stats().total_samples == 0
    assert len(ex.get_coarse_stats()) == 8
    assert isinstance(ex.export_binary(), bytes)


@pytest.fixture(scope="module")
def addon_diagnostics(lr):
    if not os.path.exists(REF_ADDON):
        pytest.skip("the add-on's diagnostics.py is not present here")
    spec = importlib.util.spec_from_file_location("lucid_addon_diagnostics", REF_ADDON)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_addon_manager_full_workflow(lr, addon_diagnostics):
    """test_diagnostics_python.py TestDiagnosticsManager.test_full_workflow,
    re-expressed: the add-on's DiagnosticsManager constructs
    lucidrenderer.DiagnosticPathTracer(width, height, config) unchanged."""
    m = addon_diagnostics.DiagnosticsManager.standard(64, 64)
    assert m.is_available
    m.enable()
    film = m.get_film()
    rec = lr.PathDiagnosticRecorder()
    rec.begin_path()
    rec.record_vertex(0, 0, lr.BsdfType.Diffuse, False, False)
    rec.record_emissive_hit(1, 0)
    film.record_path(10, 10, rec.end_path(1.5, 1.5, 1.5))
    report = m.get_report(top_n=5)
    assert report is not None
    assert report.width == 64 and report.height == 64
    assert report.global_stats.total_samples >= 1
    assert m.estimate_memory_mb() > 0
    m.disable()
    assert not m.is_enabled


def test_addon_manager_export_binary_and_clear(lr, addon_diagnostics):
    m = addon_diagnostics.DiagnosticsManager.minimal(32, 32)
    film = m.get_film()
    rec = lr.PathDiagnosticRecorder()
    rec.begin_path()
    rec.record_vertex(0, 0, lr.BsdfType.Glossy, False, False)
    film.record_path(5, 5, rec.end_path_lum(0.5))
    data = m.export_binary()
    assert data is not None and len(data) > 0
    m.clear()
    assert m.get_report().global_stats.total_samples == 0


# ---------------------------------------------------------------- against the reference film
def _path_stream(seed, n, w, h):
    """Seeded paths: repeated structures (so groups accumulate), more than 16
    distinct structures per cell (so groups are evicted), paths longer than
    16 vertices, every terminal kind, and rare bright outliers."""
    rng = np.random.default_rng(seed)
    protos = []
    for _ in range(60):
        d = int(rng.integers(0, 19))
        verts = [(int(rng.integers(-1, 6)), int(rng.integers(-1, 3)), int(rng.integers(0, 4)),
                  bool(rng.integers(0, 2)), bool(rng.random() < 0.4)) for _ in range(d)]
        term = int(rng.integers(0, 4))   # 0 none, 1 environment, 2 light, 3 emissive
        extra = (int(rng.integers(0, 5)), int(rng.integers(0, 7))) if term == 2 else \
            (int(rng.integers(0, 6)), int(rng.integers(-1, 3))) if term == 3 else None
        protos.append((verts, term, extra))
    hot = [(int(rng.integers(0, w)), int(rng.integers(0, h))) for _ in range(4)]
    for i in range(n):
        x, y = hot[i % 4] if rng.random() < 0.5 else (int(rng.integers(0, w + 3)), int(rng.integers(0, h + 3)))
        verts, term, extra = protos[int(rng.integers(0, len(protos)))]
        c = rng.random(3).astype(np.float32) * (40.0 if rng.random() < 0.03 else 1.0)
        yield x, y, verts, term, extra, [float(v) for v in c]


def _feed(sinks, stream, lr):
    for x, y, verts, term, extra, c in stream:
        for kind, s in sinks:
            s.begin_path()
            for (obj, mat, bsdf, delta, ls) in verts:
                s.record_vertex(obj, mat, lr.BsdfType(bsdf) if kind == "module" else bsdf, delta, ls)
            if term == 1:
                s.record_environment_hit()
            elif term == 2:
                s.record_light_hit(extra[0], lr.LightSourceType(extra[1]) if kind == "module" else extra[1])
            elif term == 3:
                s.record_emissive_hit(extra[0], extra[1])
        yield x, y, c


@pytest.mark.parametrize("w,h,subsample,n", [(37, 29, 2, 4000), (20, 12, 1, 3000)])
def test_standalone_film_equals_reference_film(lr, w, h, subsample, n):
    import ref_ctypes
    path = os.path.join(ref_ctypes.REF_DIR, "libref_check.so")
    if os.path.isdir(ref_ctypes.REF_SOURCES):
        ref_ctypes.build()
    if not os.path.exists(path):
        pytest.skip("reference sources absent and the reference library not built")
    cfg = lr.PathRecordingConfig.standard()
    cfg.subsample_factor = subsample
    ref = ref_ctypes.ReferenceFilm(w, h, subsample=subsample)
    film = lr.DiagnosticFilm(w, h, cfg)
    rec = lr.PathDiagnosticRecorder()
    for x, y, c in _feed([("ref", ref), ("module", rec)], _path_stream(7 + subsample, n, w, h), lr):
        ref.end_path_into_film(x, y, *c)
        film.record_path(x, y, rec.end_path(*c))
    want = ref.report(top_n=12)
    ex = lr.DiagnosticExporter(film)

    assert [film.width(), film.height(), film.sampled_width(), film.sampled_height(),
            film.total_paths_recorded()] == [want["width"], want["height"], want["sampled_width"],
                                             want["sampled_height"], want["total_paths_recorded"]]
    g = ex.get_global_stats()
    assert [g.total_samples, g.active_pixels, g.total_groups, g.total_overflow] == want["global"]
    assert want["global"][3] > 0, "the stream must overflow some cells' group tables"

    def groups(v):
        return [{"x": e.pixel_x, "y": e.pixel_y, "signature": e.signature, "count": e.sample_count,
                 "mean_luminance": e.mean_luminance, "variance_luminance": e.variance_luminance,
                 "mean_rgb": list(e.mean_rgb), "variance_rgb": list(e.variance_rgb), "depth": e.depth,
                 "coarse_type": e.coarse_type, "coarse_type_name": e.coarse_type_name} for e in v]

    def f32(o):   # JSON doubles of FP32 values back to FP32 for exact comparison
        if isinstance(o, float):
            return float(np.float32(o))
        if isinstance(o, list):
            return [f32(v) for v in o]
        if isinstance(o, dict):
            return {k: f32(v) for k, v in o.items()}
        return o

    assert groups(ex.get_top_variance_groups(12)) == f32(want["top_variance"])
    assert groups(ex.get_top_mean_groups(12)) == f32(want["top_mean"])
    got_coarse = [{"type_id": c.type_id, "name": c.name, "count": c.sample_count, "mean_luminance": c.mean_luminance,
                   "variance_luminance": c.variance_luminance, "mean_rgb": list(c.mean_rgb),
                   "variance_rgb": list(c.variance_rgb)} for c in ex.get_coarse_stats()]
    assert got_coarse == f32(want["coarse"])
    assert [{"category": s.category, "severity": s.severity, "message": s.message, "action": s.action}
            for s in ex.generate_suggestions()] == want["suggestions"]
    assert ex.export_metadata_json() == want["metadata_json"] == film.metadata_json()
    assert list(ex.export_binary()) == want["binary"]


@pytest.mark.parametrize("w,h,subsample,n", [(37, 29, 2, 4000)])
def test_standalone_film_cells_equal_reference_cells(lr, w, h, subsample, n):
    """Cell by cell, through the C ABI (lucid_diag_film_*)."""
    import lucid_capi
    import ref_ctypes
    path = os.path.join(ref_ctypes.REF_DIR, "libref_check.so")
    if not os.path.exists(path):
        pytest.skip("the reference library is not built")
    ref = ref_ctypes.ReferenceFilm(w, h, subsample=subsample)
    film = lucid_capi.DiagFilm(w, h, subsample=subsample)

    class CtypesRecorder:   # PathDiagnosticRecorder over a LucidPathTrace
        def begin_path(self):
            self.t = lucid_capi.PathTrace()

        def _push(self, obj, mat, bsdf, flags):
            if self.t.depth >= 16:
                return False
            v = self.t.vertices[self.t.depth]
            v.object_id, v.material_id, v.bsdf_type, v.flags = obj, mat, bsdf, flags
            self.t.depth += 1
            return True

        def record_vertex(self, obj, mat, bsdf, delta, ls):
            self._push(obj, mat, bsdf, (1 if delta else 0) | (2 if ls else 0))

        def record_environment_hit(self):
            if self._push(-1, -1, 5, 0):
                self.t.light_type = 5

        def record_light_hit(self, lid, lt):
            if self._push(-(lid + 2), -1, 4, 0):
                self.t.light_type = lt

        def record_emissive_hit(self, obj, mat):
            if self._push(obj, mat, 4, 0):
                self.t.light_type = 6

    rec = CtypesRecorder()
    hashes_equal = 0
    for x, y, c in _feed([("ref", ref), ("ctypes", rec)], _path_stream(11, n, w, h), lr):
        want_hash = ref.end_path_into_film(x, y, *c)
        rec.t.contribution[:] = c
        assert film.lib.lucid_path_trace_hash(rec.t) == want_hash
        hashes_equal += 1
        film.record_path(x, y, rec.t)
    assert hashes_equal == n
    want = ref.report()
    cells = want["cells"]
    sw, sh = want["sampled_width"], want["sampled_height"]
    assert len(cells) == sw * sh
    for sy in range(sh):
        for sx in range(sw):
            total, ngroups, overflow, outliers, hs = cells[sy * sw + sx]
            info, groups = film.pixel(sx * subsample, sy * subsample)
            assert (int(info["sample_count"]), int(info["group_count"]), int(info["overflow_count"]),
                    int(info["outlier_count"])) == (total, ngroups, overflow, outliers), (sx, sy)
            assert sorted((int(g["hash"]), int(g["count"])) for g in groups) == \
                sorted((int(hh), int(cnt)) for hh, cnt in hs), (sx, sy)
