"""ctypes binding of the Lucid reference's own render path built here
(oracle/_ref/libref_*.so, `make -C oracle ref`: the reference's unmodified
headers and node evaluator against the project-written mp-units shim).

TEST INFRASTRUCTURE ONLY: the pin of the oracle (tests/test_reference_pin.py)
and the timed CPU baseline of bench.py --impl reference.  The product never
imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
REF_SOURCES = "/root/reference/LucidRenderer/cpp_renderer"

_libs: dict = {}


def build() -> bool:
    """Build the reference libraries when the reference sources are present
    (they are not on machines that only receive the built files)."""
    if not os.path.isdir(REF_SOURCES):
        return False
    subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={REF_SOURCES}"])
    return True


def _host_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def bench_library_path() -> str | None:
    """The reference built with its own flags (-O3 -march=native -ffast-math
    -flto): the -march=native build when this host has every CPU feature of
    the machine that built it, else the x86-64-v3 build."""
    native = os.path.join(REF_DIR, "libref_bench.so")
    flags = os.path.join(REF_DIR, "libref_bench.cpuflags")
    portable = os.path.join(REF_DIR, "libref_bench_x86-64-v3.so")
    if os.path.exists(native) and os.path.exists(flags):
        with open(flags) as f:
            need = set(f.read().split())
        if need <= _host_flags():
            return native
    return portable if os.path.exists(portable) else None


def load(path: str) -> ctypes.CDLL:
    if path not in _libs:
        lib = ctypes.CDLL(path)
        f, i, p = ctypes.c_float, ctypes.c_int, ctypes.c_void_p
        for name, (res, args) in {
            "ref_create": (p, []), "ref_destroy": (None, [p]), "ref_load_scene_json": (i, [p, ctypes.c_char_p]),
            "ref_set_camera": (None, [p] + [f] * 10), "ref_set_algorithm": (None, [p, ctypes.c_char_p]),
            "ref_render_tile": (i, [p] + [i] * 9 + [p]),
            "ref_render_debug": (i, [p] + [i] * 6 + [ctypes.c_char_p, p]), "ref_max_threads": (i, []),
            "ref_film_create": (p, [ctypes.c_longlong, ctypes.c_longlong, i, i, i, i, f, f]),
            "ref_film_destroy": (None, [p]), "ref_film_clear": (None, [p]),
            "ref_recorder_create": (p, []), "ref_recorder_destroy": (None, [p]), "ref_recorder_begin": (None, [p]),
            "ref_recorder_vertex": (None, [p, i, i, i, i, i]), "ref_recorder_environment": (None, [p]),
            "ref_recorder_light": (None, [p, i, i]), "ref_recorder_emissive": (None, [p, i, i]),
            "ref_recorder_end_into": (ctypes.c_ulonglong, [p, p, ctypes.c_longlong, ctypes.c_longlong, f, f, f]),
            "ref_film_report": (ctypes.c_void_p, [p, i, i]), "ref_free": (None, [ctypes.c_void_p]),
            "ref_enable_diagnostics": (None, [p, i, i, i, i, f, f]), "ref_disable_diagnostics": (None, [p]),
            "ref_diag_report": (ctypes.c_void_p, [p, i, i, i]), "ref_set_threads": (None, [i]),
        }.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _libs[path] = lib
    return _libs[path]


class ReferenceRenderer:
    """The reference's PyRenderer (render_tile, render_debug) through the C
    driver in oracle/ref_driver.cpp."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(REF_DIR, "libref_check.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = load(path)
        self.h = self.lib.ref_create()

    def __del__(self):
        try:
            self.lib.ref_destroy(self.h)
        except Exception:
            pass

    def threads(self) -> int:
        return int(self.lib.ref_max_threads())

    def set_threads(self, n: int):
        """OpenMP threads of the render loops (0: all processors); process-wide."""
        self.lib.ref_set_threads(n)

    def load_scene_json(self, text: str) -> bool:
        return bool(self.lib.ref_load_scene_json(self.h, text.encode()))

    def set_camera(self, *cam):
        self.lib.ref_set_camera(self.h, *[float(c) for c in cam])

    def set_algorithm(self, name: str):
        self.lib.ref_set_algorithm(self.h, name.encode())

    def render(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
               tile_x=0, tile_y=0) -> np.ndarray:
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        out = np.zeros((tile_h, tile_w, 4), np.float32)
        rc = self.lib.ref_render_tile(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples,
                                      sample_offset, max_depth, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference render_tile returned a buffer of the wrong size")
        return out

    def enable_diagnostics(self, subsample=2, max_groups=16, max_outliers=4, max_depth=16,
                           variance_threshold=0.001, outlier_threshold=3.0):
        self.lib.ref_enable_diagnostics(self.h, subsample, max_groups, max_outliers, max_depth,
                                        variance_threshold, outlier_threshold)

    def disable_diagnostics(self):
        self.lib.ref_disable_diagnostics(self.h)

    def diag_report(self, tile_w, tile_h, top_n=10) -> dict:
        """get_diagnostic_stats, get_pixel_diagnostic of every tile pixel (groups
        sorted by variance), get_top_variance_groups and export_diagnostic_json
        of the last diagnostic render."""
        import json
        c = self.lib.ref_diag_report(self.h, tile_w, tile_h, top_n)
        try:
            return json.loads(ctypes.string_at(c).decode())
        finally:
            self.lib.ref_free(c)

    def render_debug(self, mode: str, tile_w, tile_h, full_w=None, full_h=None, tile_x=0, tile_y=0) -> np.ndarray:
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        out = np.zeros((tile_h, tile_w, 4), np.float32)
        rc = self.lib.ref_render_debug(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, mode.encode(),
                                       out.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference render_debug returned a buffer of the wrong size")
        return out


class ReferenceFilm:
    """The reference's DiagnosticFilm with a PathDiagnosticRecorder feeding it
    and a DiagnosticExporter reading it (diagnostics/*.hpp)."""

    def __init__(self, width, height, subsample=2, max_groups=16, max_outliers=4, max_depth=16,
                 variance_threshold=0.001, outlier_threshold=3.0, path: str | None = None):
        path = path or os.path.join(REF_DIR, "libref_check.so")
        self.lib = load(path)
        self.subsample = subsample
        self.f = self.lib.ref_film_create(width, height, subsample, max_groups, max_outliers, max_depth,
                                          variance_threshold, outlier_threshold)
        self.r = self.lib.ref_recorder_create()

    def __del__(self):
        try:
            self.lib.ref_recorder_destroy(self.r)
            self.lib.ref_film_destroy(self.f)
        except Exception:
            pass

    # PathDiagnosticRecorder calls
    def begin_path(self):
        self.lib.ref_recorder_begin(self.r)

    def record_vertex(self, obj, mat, bsdf, delta, light_sampled):
        self.lib.ref_recorder_vertex(self.r, obj, mat, bsdf, int(delta), int(light_sampled))

    def record_environment_hit(self):
        self.lib.ref_recorder_environment(self.r)

    def record_light_hit(self, light_id, light_type):
        self.lib.ref_recorder_light(self.r, light_id, light_type)

    def record_emissive_hit(self, obj, mat):
        self.lib.ref_recorder_emissive(self.r, obj, mat)

    def end_path_into_film(self, x, y, r, g, b) -> int:
        return int(self.lib.ref_recorder_end_into(self.r, self.f, x, y, r, g, b))

    def clear(self):
        self.lib.ref_film_clear(self.f)

    def report(self, top_n: int = 10) -> dict:
        import json
        c = self.lib.ref_film_report(self.f, top_n, self.subsample)
        try:
            return json.loads(ctypes.string_at(c).decode())
        finally:
            self.lib.ref_free(c)

