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

    def render_debug(self, mode: str, tile_w, tile_h, full_w=None, full_h=None, tile_x=0, tile_y=0) -> np.ndarray:
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        out = np.zeros((tile_h, tile_w, 4), np.float32)
        rc = self.lib.ref_render_debug(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, mode.encode(),
                                       out.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference render_debug returned a buffer of the wrong size")
        return out
