"""ctypes binding of the CPU oracle (oracle/_build/liblucid_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker and the timed CPU
baseline.  The product never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liblucid_oracle.so")

# Same layout as LucidSampleRecord (include/lucid_cuda.h) and orc::SampleRec.
RECORD_DTYPE = np.dtype([("rgb", np.float32, 3), ("primary_mesh", np.int32), ("primary_tri", np.int32),
                         ("bounces", np.uint32), ("nee_tests", np.uint32), ("nee_occluded", np.uint32),
                         ("hash", np.uint64)], align=True)

_lib = None


def build() -> None:
    subprocess.check_call(["make", "-s", "-C", HERE])


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        f, i, p, u = ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32
        sig = {
            "orc_create": (p, []), "orc_destroy": (None, [p]), "orc_set_options": (None, [i, i]),
            "orc_set_draw_order": (None, [i]),
            "orc_load_scene_json": (i, [p, ctypes.c_char_p]), "orc_set_camera": (None, [p] + [f] * 10),
            "orc_set_algorithm": (None, [p, ctypes.c_char_p]),
            "orc_render_tile": (i, [p, i, i, i, i, i, i, i, i, i, p, p, i]),
            "orc_render_debug": (i, [p, i, i, i, i, i, i, i, p]),
            "orc_scene_stats": (None, [p, p]), "orc_scene_lights": (i, [p, p, p, p, i]),
            "orc_closest_hit": (None, [p, p, p, f, f, p, p, p]),
            "orc_sizeof_record": (u, []), "orc_fresnel_schlick": (f, [f, f]), "orc_fresnel_dielectric": (f, [f, f]),
            "orc_ggx_d": (f, [f, f]), "orc_ggx_g1": (f, [f, f]), "orc_ggx_g2": (f, [f, f, f]),
            "orc_mis_power": (f, [f, f]), "orc_pdfw_from_area": (f, [f, f, f]), "orc_inv_sq": (f, [f]),
            "orc_hg_eval": (f, [f, f]), "orc_hg_sample": (None, [f, p, f, f, p, p]),
            "orc_rng_sequence": (None, [u, u, u, i, p, p]), "orc_isect_tri": (i, [p, p, p, f, f, p]),
            "orc_isect_aabb": (i, [p, p, p, p]), "orc_isect_sphere": (i, [p, p, p, f, p]),
            "orc_eval_bsdf": (None, [p, p, p, p, p, p]),
            "orc_sample_bsdf": (i, [p, p, p, f, f, f, u, u, u, p, p, p, p, p]), "orc_lm": (f, [i, f]),
            "orc_render_tile_diag": (i, [p, i, i, i, i, i, i, i, i, i, i, p, i]),
            "orc_diag_pixel": (i, [p, i, i, i, p, p, i]), "orc_diag_stats": (None, [p, p]),
            "orc_diag_top_groups": (i, [p, i, i, p, p, i]),
            "orc_diag_coarse": (None, [p, p]), "orc_diag_suggestions": (i, [p, p, i]),
            "orc_diag_export_binary": (ctypes.c_longlong, [p, i, i, p, ctypes.c_size_t]),
            "orc_render_tile_f64": (i, [p, i, i, i, i, i, i, i, i, i, p, i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        assert lib.orc_sizeof_record() == RECORD_DTYPE.itemsize
        _lib = lib
    return _lib


# Same layouts as LucidDiagGroup / LucidDiagPixel (include/lucid_cuda.h).
DIAG_GROUP_DTYPE = np.dtype([("hash", np.uint64), ("count", np.uint32), ("depth", np.uint8),
                             ("coarse_type", np.uint8), ("light_type", np.uint8), ("strategy", np.uint8),
                             ("mean_rgb", np.float32, 3), ("variance_rgb", np.float32, 3),
                             ("mean_luminance", np.float32), ("total_variance", np.float32),
                             ("object_ids", np.int32, 16), ("bsdf", np.uint8, 16), ("flags", np.uint8, 16),
                             ("positions", np.float32, (16, 3)), ("normals", np.float32, (16, 3))], align=True)
DIAG_PIXEL_DTYPE = np.dtype([("valid", np.int32), ("sample_count", np.uint32), ("group_count", np.uint32),
                             ("outlier_count", np.uint32), ("overflow_count", np.uint32), ("variance", np.float32),
                             ("mean_rgb", np.float32, 3)], align=True)


def fptr(a: np.ndarray):
    return a.ctypes.data


class OrcCoarse(ctypes.Structure):
    _fields_ = [("type_id", ctypes.c_int32), ("name", ctypes.c_char * 32), ("sample_count", ctypes.c_uint64),
                ("mean_luminance", ctypes.c_float), ("variance_luminance", ctypes.c_float),
                ("mean_rgb", ctypes.c_float * 3), ("variance_rgb", ctypes.c_float * 3)]


class Oracle:
    """The reference's PyRenderer surface, restated on the CPU."""

    def __init__(self, device_math: bool = True, canonical_ties: bool = True, draw_rtl: bool = False):
        self.lib = load()
        self.lib.orc_set_options(int(device_math), int(canonical_ties))
        self.lib.orc_set_draw_order(int(draw_rtl))
        self.h = self.lib.orc_create()

    def __del__(self):
        try:
            self.lib.orc_destroy(self.h)
        except Exception:
            pass

    def set_options(self, device_math: bool = True, canonical_ties: bool = True):
        self.lib.orc_set_options(int(device_math), int(canonical_ties))

    def load_scene_json(self, text: str) -> bool:
        return bool(self.lib.orc_load_scene_json(self.h, text.encode()))

    def set_camera(self, *cam):
        self.lib.orc_set_camera(self.h, *[float(c) for c in cam])

    def set_algorithm(self, name: str):
        self.lib.orc_set_algorithm(self.h, name.encode())

    def render(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
               tile_x=0, tile_y=0, records=False, threads=0):
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        img = np.zeros((tile_h, tile_w, 4), np.float32)
        recs = np.zeros(tile_w * tile_h * samples, RECORD_DTYPE) if records else None
        rc = self.lib.orc_render_tile(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples,
                                      sample_offset, max_depth, fptr(img),
                                      fptr(recs) if recs is not None else None, threads)
        return img, recs, rc

    def render_f64(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
                   tile_x=0, tile_y=0, threads=0):
        """Per-pixel FP64 sum of the samples' FP32 radiance (clamp >= 0, Y-flipped)."""
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        img = np.zeros((tile_h, tile_w, 4), np.float64)
        rc = self.lib.orc_render_tile_f64(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples,
                                          sample_offset, max_depth, fptr(img), threads)
        return img, rc

    def render_debug(self, mode: int, tile_w, tile_h, full_w=None, full_h=None, tile_x=0, tile_y=0):
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        img = np.zeros((tile_h, tile_w, 4), np.float32)
        self.lib.orc_render_debug(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, mode, fptr(img))
        return img

    def render_diag(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
                    tile_x=0, tile_y=0, subsample=2, threads=0):
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        img = np.zeros((tile_h, tile_w, 4), np.float32)
        rc = self.lib.orc_render_tile_diag(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples,
                                           sample_offset, max_depth, subsample, fptr(img), threads)
        return img, rc

    def diag_pixel(self, x, y, sort_by_mean=False, cap=32):
        info = np.zeros(1, DIAG_PIXEL_DTYPE)
        groups = np.zeros(cap, DIAG_GROUP_DTYPE)
        n = self.lib.orc_diag_pixel(self.h, x, y, int(sort_by_mean), fptr(info), fptr(groups), cap)
        return info[0], groups[:n]

    def diag_top_groups(self, n, by_mean=False):
        groups = np.zeros(max(n, 1), DIAG_GROUP_DTYPE)
        xy = np.zeros((max(n, 1), 2), np.int32)
        m = self.lib.orc_diag_top_groups(self.h, n, int(by_mean), fptr(groups), fptr(xy), groups.size)
        return groups[:m], xy[:m]

    def diag_coarse(self):
        """get_coarse_stats: eight (type_id, name, count, mean_lum, var_lum, mean_rgb, var_rgb)."""
        out = (OrcCoarse * 8)()
        self.lib.orc_diag_coarse(self.h, ctypes.addressof(out))
        return [(c.type_id, c.name.decode(), c.sample_count, c.mean_luminance, c.variance_luminance,
                 tuple(c.mean_rgb), tuple(c.variance_rgb)) for c in out]

    def diag_suggestion_kinds(self):
        """generate_suggestions as kinds: 0 glossy, 1 indirect, 2 diffuse, 3 capacity."""
        out = np.zeros(8, np.int32)
        n = self.lib.orc_diag_suggestions(self.h, fptr(out), 8)
        return out[:n].tolist()

    def diag_export_binary(self, max_groups=16, max_outliers=4) -> bytes:
        n = self.lib.orc_diag_export_binary(self.h, max_groups, max_outliers, None, 0)
        buf = np.zeros(max(n, 1), np.uint8)
        self.lib.orc_diag_export_binary(self.h, max_groups, max_outliers, fptr(buf), buf.size)
        return buf[:n].tobytes()

    def diag_stats(self):
        out = np.zeros(5, np.uint64)
        self.lib.orc_diag_stats(self.h, fptr(out))
        return out.tolist()

    def scene_stats(self):
        out = np.zeros(6, np.int32)
        self.lib.orc_scene_stats(self.h, fptr(out))
        return out.tolist()

    def scene_lights(self, cap=1 << 16):
        cdf = np.zeros(cap, np.float32)
        area = np.zeros(cap, np.float32)
        em = np.zeros((cap, 3), np.float32)
        n = self.lib.orc_scene_lights(self.h, fptr(cdf), fptr(area), fptr(em), cap)
        return cdf[:n].copy(), area[:n].copy(), em[:n].copy()
