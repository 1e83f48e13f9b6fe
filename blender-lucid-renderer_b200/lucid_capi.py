"""ctypes binding of liblucid_cuda.so (the C ABI in include/lucid_cuda.h).

This is the reference-facing boundary as a non-pybind caller sees it (the
same stub a ctypes/cffi integration would use).  Importing it fails loudly
when the CUDA library has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblucid_cuda.so")

LUCID_OK = 0
LUCID_ERR_NO_SCENE = -1
LUCID_ERR_OOM = -2
LUCID_ERR_TIMEOUT = -3
LUCID_ERR_CANCELLED = -4
LUCID_ERR_INVALID = -5
LUCID_ERR_CUDA = -6
LUCID_ERR_OVERFLOW = -7
LUCID_RENDER_PROFILE = 1


class RenderParams(ctypes.Structure):
    _fields_ = [("tile_x", ctypes.c_int), ("tile_y", ctypes.c_int), ("tile_w", ctypes.c_int),
                ("tile_h", ctypes.c_int), ("full_w", ctypes.c_int), ("full_h", ctypes.c_int),
                ("samples", ctypes.c_int), ("sample_offset", ctypes.c_int), ("max_depth", ctypes.c_int),
                ("flags", ctypes.c_int)]


_F3 = ctypes.c_float * 3


class MeshDesc(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("num_vertices", ctypes.c_int32), ("triangles", ctypes.c_void_p),
                ("num_triangles", ctypes.c_int32), ("triangle_normals", ctypes.c_void_p), ("smooth", ctypes.c_int32),
                ("base_color", _F3), ("metallic", ctypes.c_float), ("roughness", ctypes.c_float), ("emission", _F3),
                ("transmission", ctypes.c_float), ("ior", ctypes.c_float), ("surface", ctypes.c_int32),
                ("volume_density", ctypes.c_float), ("volume_anisotropy", ctypes.c_float), ("volume_color", _F3),
                ("volume_absorption", _F3), ("volume_dims", ctypes.c_int32 * 3), ("volume_world_min", _F3),
                ("volume_world_max", _F3), ("volume_grid", ctypes.c_void_p)]


class LightDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int32), ("position", _F3), ("direction", _F3), ("color", _F3),
                ("energy", ctypes.c_float), ("radius", ctypes.c_float), ("spot_size", ctypes.c_float),
                ("spot_blend", ctypes.c_float), ("size", ctypes.c_float), ("size_y", ctypes.c_float),
                ("shape", ctypes.c_int32), ("right", _F3), ("up", _F3)]


LUCID_EDIT_MATERIAL = 1
LUCID_EDIT_LIGHT = 2


class SceneEdit(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("index", ctypes.c_int32), ("base_color", _F3), ("metallic", ctypes.c_float),
                ("roughness", ctypes.c_float), ("emission", _F3), ("transmission", ctypes.c_float),
                ("ior", ctypes.c_float), ("light", LightDesc)]


def _light_desc(l: dict, d: LightDesc) -> None:
    d.type = int(l["type"])
    d.position, d.direction, d.color = _F3(*l["position"]), _F3(*l["direction"]), _F3(*l["color"])
    d.energy, d.radius = float(l["energy"]), float(l["radius"])
    d.spot_size, d.spot_blend = float(l["spot_size"]), float(l["spot_blend"])
    d.size, d.size_y, d.shape = float(l["size"]), float(l["size_y"]), int(l["shape"])
    d.right, d.up = _F3(*l["right"]), _F3(*l["up"])


def scene_edits(edits) -> ctypes.Array:
    """LucidSceneEdit array from dicts: {"mesh": i, "material": {base_color,
    metallic, roughness, emission, transmission, ior}} or {"light": j,
    "desc": a light of lucid_scenes.scene_arrays(...)["lights"]}."""
    arr = (SceneEdit * max(1, len(edits)))()
    for i, e in enumerate(edits):
        x = arr[i]
        if "mesh" in e:
            m = e["material"]
            x.kind, x.index = LUCID_EDIT_MATERIAL, int(e["mesh"])
            x.base_color, x.emission = _F3(*m["base_color"]), _F3(*m["emission"])
            x.metallic, x.roughness = float(m["metallic"]), float(m["roughness"])
            x.transmission, x.ior = float(m["transmission"]), float(m["ior"])
        else:
            x.kind, x.index = LUCID_EDIT_LIGHT, int(e["light"])
            _light_desc(e["desc"], x.light)
    return arr


class SceneDesc(ctypes.Structure):
    _fields_ = [("meshes", ctypes.c_void_p), ("num_meshes", ctypes.c_int32), ("lights", ctypes.c_void_p),
                ("num_lights", ctypes.c_int32), ("environment", _F3)]


def _scene_desc(arrays: dict):
    """ctypes descriptors for lucid_scenes.scene_arrays output; returns the
    descriptor and the objects that must stay alive while it is used."""
    keep = []

    def ptr(a, dtype):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a.ctypes.data

    ms = (MeshDesc * max(1, len(arrays["meshes"])))()
    for i, m in enumerate(arrays["meshes"]):
        d = ms[i]
        d.vertices = ptr(m["vertices"], np.float32)
        d.num_vertices = len(m["vertices"]) // 3
        d.triangles = ptr(m["triangles"], np.int32)
        d.num_triangles = len(m["triangles"]) // 3
        d.triangle_normals = ptr(m["triangle_normals"], np.float32)
        d.smooth = int(m["smooth"])
        d.base_color = _F3(*m["base_color"])
        d.metallic, d.roughness = float(m["metallic"]), float(m["roughness"])
        d.emission = _F3(*m["emission"])
        d.transmission, d.ior = float(m["transmission"]), float(m["ior"])
        d.surface = int(m["surface"])
        d.volume_density, d.volume_anisotropy = float(m["volume_density"]), float(m["volume_anisotropy"])
        d.volume_color, d.volume_absorption = _F3(*m["volume_color"]), _F3(*m["volume_absorption"])
        d.volume_dims = (ctypes.c_int32 * 3)(*m["volume_dims"])
        d.volume_world_min, d.volume_world_max = _F3(*m["volume_world_min"]), _F3(*m["volume_world_max"])
        d.volume_grid = ptr(m["volume_grid"], np.float32)
    ls_ = (LightDesc * max(1, len(arrays["lights"])))()
    for i, l in enumerate(arrays["lights"]):
        _light_desc(l, ls_[i])
    keep += [ms, ls_]
    sd = SceneDesc(ctypes.addressof(ms), len(arrays["meshes"]), ctypes.addressof(ls_), len(arrays["lights"]),
                   _F3(*arrays["environment"]))
    return sd, keep


class DiagCoarse(ctypes.Structure):
    _fields_ = [("type_id", ctypes.c_int32), ("name", ctypes.c_char * 32), ("sample_count", ctypes.c_uint64),
                ("mean_luminance", ctypes.c_float), ("variance_luminance", ctypes.c_float),
                ("mean_rgb", ctypes.c_float * 3), ("variance_rgb", ctypes.c_float * 3)]


class DiagSuggestion(ctypes.Structure):
    _fields_ = [("category", ctypes.c_char * 16), ("severity", ctypes.c_char * 16), ("message", ctypes.c_char * 128),
                ("action", ctypes.c_char * 128)]


class SampleRecord(ctypes.Structure):
    _fields_ = [("rgb", ctypes.c_float * 3), ("primary_mesh", ctypes.c_int32), ("primary_tri", ctypes.c_int32),
                ("bounces", ctypes.c_uint32), ("nee_tests", ctypes.c_uint32), ("nee_occluded", ctypes.c_uint32),
                ("hash", ctypes.c_uint64)]


RECORD_DTYPE = np.dtype([("rgb", np.float32, 3), ("primary_mesh", np.int32), ("primary_tri", np.int32),
                         ("bounces", np.uint32), ("nee_tests", np.uint32), ("nee_occluded", np.uint32),
                         ("hash", np.uint64)], align=True)
assert RECORD_DTYPE.itemsize == ctypes.sizeof(SampleRecord)


class KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int), ("total_ms", ctypes.c_double),
                ("algo_bytes", ctypes.c_double), ("units", ctypes.c_double)]


class RenderStats(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_double), ("paths", ctypes.c_double), ("segments", ctypes.c_double),
                ("shadow_rays", ctypes.c_double), ("waves", ctypes.c_int), ("num_kinds", ctypes.c_int),
                ("kinds", KernelStat * 12)]


class DiagConfig(ctypes.Structure):
    _fields_ = [("subsample_factor", ctypes.c_int), ("max_groups_per_pixel", ctypes.c_int),
                ("max_outliers_per_pixel", ctypes.c_int), ("max_depth", ctypes.c_int),
                ("variance_threshold", ctypes.c_float), ("outlier_threshold", ctypes.c_float),
                ("record_capacity", ctypes.c_longlong)]


class PathVertex(ctypes.Structure):
    _fields_ = [("object_id", ctypes.c_int32), ("material_id", ctypes.c_int16), ("bsdf_type", ctypes.c_uint8),
                ("flags", ctypes.c_uint8)]


class PathTrace(ctypes.Structure):
    """LucidPathTrace (include/lucid_cuda.h): PathTrace of path_types.hpp:249-257."""
    _fields_ = [("vertices", PathVertex * 16), ("positions", (ctypes.c_float * 3) * 16),
                ("normals", (ctypes.c_float * 3) * 16), ("depth", ctypes.c_uint32),
                ("contribution", ctypes.c_float * 3), ("light_type", ctypes.c_uint8), ("strategy", ctypes.c_uint8),
                ("pad", ctypes.c_uint8 * 2)]


# LucidDiagGroup / LucidDiagPixel / LucidDiagStats (include/lucid_cuda.h).
DIAG_GROUP_DTYPE = np.dtype([("hash", np.uint64), ("count", np.uint32), ("depth", np.uint8),
                             ("coarse_type", np.uint8), ("light_type", np.uint8), ("strategy", np.uint8),
                             ("mean_rgb", np.float32, 3), ("variance_rgb", np.float32, 3),
                             ("mean_luminance", np.float32), ("total_variance", np.float32),
                             ("object_ids", np.int32, 16), ("bsdf", np.uint8, 16), ("flags", np.uint8, 16),
                             ("positions", np.float32, (16, 3)), ("normals", np.float32, (16, 3))], align=True)
DIAG_PIXEL_DTYPE = np.dtype([("valid", np.int32), ("sample_count", np.uint32), ("group_count", np.uint32),
                             ("outlier_count", np.uint32), ("overflow_count", np.uint32), ("variance", np.float32),
                             ("mean_rgb", np.float32, 3)], align=True)
DIAG_STATS_FIELDS = ("total_samples", "active_pixels", "total_groups", "total_overflow", "paths_recorded")


class JobDesc(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_int), ("camera", ctypes.c_float * 10), ("algorithm", ctypes.c_char * 16),
                ("width", ctypes.c_int), ("height", ctypes.c_int), ("samples", ctypes.c_int),
                ("max_depth", ctypes.c_int), ("interactive", ctypes.c_int), ("guided", ctypes.c_int),
                ("guide_seed", ctypes.c_int)]


class BatchJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("camera", ctypes.c_float * 10), ("params", RenderParams),
                ("out_rgba", ctypes.c_void_p)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int), ("done", ctypes.c_int), ("refused", ctypes.c_int),
                ("running", ctypes.c_int), ("queued", ctypes.c_int),
                ("latency_p50_ms", ctypes.c_double), ("latency_p99_ms", ctypes.c_double),
                ("first_p50_ms", ctypes.c_double), ("first_p99_ms", ctypes.c_double),
                ("samples_per_s", ctypes.c_double), ("bytes_reserved", ctypes.c_longlong),
                ("bytes_running", ctypes.c_longlong), ("budget_bytes", ctypes.c_longlong),
                ("batches", ctypes.c_int), ("batched_jobs", ctypes.c_int)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_REFUSED, JOB_FAILED, JOB_CANCELLED = range(6)

# Every symbol include/lucid_cuda.h declares, with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
SIGNATURES = {
    "lucid_cuda_create": (_I, [_I, ctypes.POINTER(_P)]),
    "lucid_cuda_destroy": (None, [_P]),
    "lucid_cuda_last_error": (ctypes.c_char_p, [_P]),
    "lucid_cuda_device_info": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "lucid_cuda_load_scene_json": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t]),
    "lucid_cuda_load_scene_arrays": (_I, [_P, ctypes.c_void_p]),
    "lucid_scene_digest": (_I, [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]),
    "lucid_cuda_diag_coarse_stats": (_I, [_P, ctypes.c_void_p]),
    "lucid_cuda_diag_suggestions": (_I, [_P, ctypes.c_void_p, _I]),
    "lucid_cuda_diag_export_binary": (ctypes.c_longlong, [_P, ctypes.c_void_p, ctypes.c_size_t]),
    "lucid_cuda_diag_metadata_json": (ctypes.c_longlong, [_P, ctypes.c_void_p, ctypes.c_size_t]),
    "lucid_cuda_set_camera": (_I, [_P] + [_F] * 10),
    "lucid_cuda_set_algorithm": (_I, [_P, ctypes.c_char_p]),
    "lucid_cuda_scene_stats": (_I, [_P, ctypes.POINTER(_I)]),
    "lucid_cuda_inspect_scene": (_I, [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_I), _P, _P, _P, _I]),
    "lucid_cuda_render": (_I, [_P, ctypes.POINTER(RenderParams), _P, _P]),
    "lucid_cuda_render_device": (_I, [_P, ctypes.POINTER(RenderParams), _P]),
    "lucid_cuda_render_noalloc": (_I, [_P, ctypes.POINTER(RenderParams), _P]),
    "lucid_cuda_render_batch": (_I, [_P, _P, _I, ctypes.c_char_p]),
    "lucid_cuda_set_combining": (_I, [_P, _I]),
    "lucid_cuda_combine_stats": (_I, [_I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "lucid_cuda_render_debug": (_I, [_P, _I, _I, _I, _I, _I, _I, ctypes.c_char_p, _P]),
    "lucid_cuda_get_stats": (_I, [_P, ctypes.POINTER(RenderStats)]),
    "lucid_cuda_set_wave_capacity": (_I, [_P, ctypes.c_longlong]),
    "lucid_cuda_async_start": (_I, [_P, _I, _I, _I]),
    "lucid_cuda_async_poll": (_I, [_P, ctypes.POINTER(_I), _P, ctypes.c_size_t]),
    "lucid_cuda_async_revision": (_I, [_P]),
    "lucid_cuda_async_reset": (_I, [_P, _I, _I, _I]),
    "lucid_cuda_async_stop": (_I, [_P]),
    "lucid_cuda_async_running": (_I, [_P]),
    "lucid_cuda_render_f64": (_I, [_P, ctypes.POINTER(RenderParams), _P]),
    "lucid_cuda_diag_enable": (_I, [_P, ctypes.POINTER(DiagConfig)]),
    "lucid_cuda_diag_disable": (_I, [_P]),
    "lucid_cuda_diag_enabled": (_I, [_P]),
    "lucid_cuda_diag_clear": (_I, [_P]),
    "lucid_cuda_diag_stats": (_I, [_P, _P]),
    "lucid_cuda_diag_pixel": (_I, [_P, _I, _I, _I, _P, _P, _I]),
    "lucid_cuda_diag_variance_map": (_I, [_P, _P, ctypes.c_size_t]),
    "lucid_cuda_diag_top_groups": (_I, [_P, _I, _I, _P, _P, _I]),
    "lucid_diag_film_create": (_I, [ctypes.c_longlong, ctypes.c_longlong, ctypes.POINTER(DiagConfig),
                                    ctypes.POINTER(_P)]),
    "lucid_diag_film_destroy": (None, [_P]),
    "lucid_diag_film_record_path": (_I, [_P, ctypes.c_longlong, ctypes.c_longlong, ctypes.POINTER(PathTrace)]),
    "lucid_diag_film_clear": (_I, [_P]),
    "lucid_diag_film_info": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "lucid_diag_film_stats": (_I, [_P, _P]),
    "lucid_diag_film_pixel": (_I, [_P, ctypes.c_longlong, ctypes.c_longlong, _I, _P, _P, _I]),
    "lucid_diag_film_top_groups": (_I, [_P, _I, _I, _P, _P, _I]),
    "lucid_diag_film_coarse_stats": (_I, [_P, ctypes.c_void_p]),
    "lucid_diag_film_suggestions": (_I, [_P, ctypes.c_void_p, _I]),
    "lucid_diag_film_export_binary": (ctypes.c_longlong, [_P, ctypes.c_void_p, ctypes.c_size_t]),
    "lucid_diag_film_metadata_json": (ctypes.c_longlong, [_P, ctypes.c_void_p, ctypes.c_size_t]),
    "lucid_path_trace_hash": (ctypes.c_uint64, [ctypes.POINTER(PathTrace)]),
    "lucid_path_trace_coarse_type": (_I, [ctypes.POINTER(PathTrace)]),
    "lucid_cuda_update_scene": (_I, [_P, _P, _I]),
    "lucid_cuda_set_launch_profile": (_I, [_P, _I]),
    "lucid_server_update_scene": (_I, [_P, _I, _P, _I]),
    "lucid_server_create": (_I, [_I, _I, ctypes.c_longlong, ctypes.POINTER(_P)]),
    "lucid_server_destroy": (None, [_P]),
    "lucid_server_last_error": (ctypes.c_char_p, [_P]),
    "lucid_server_add_scene": (_I, [_P, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_I)]),
    "lucid_server_add_scene_arrays": (_I, [_P, ctypes.c_void_p, ctypes.POINTER(_I)]),
    "lucid_server_submit": (_I, [_P, ctypes.POINTER(JobDesc), ctypes.POINTER(_I)]),
    "lucid_server_job_state": (_I, [_P, _I, ctypes.POINTER(_I)]),
    "lucid_server_wait": (_I, [_P, _I, _I]),
    "lucid_server_result": (_I, [_P, _I, _P, ctypes.c_size_t]),
    "lucid_server_cancel": (_I, [_P, _I]),
    "lucid_server_stats": (_I, [_P, ctypes.POINTER(ServerStats)]),
    "lucid_server_set_batching": (_I, [_P, ctypes.c_longlong]),
    "lucid_admission_plan": (_I, [ctypes.c_longlong, ctypes.c_longlong, _I, _P, _I, _P]),
    "lucid_batch_plan": (_I, [ctypes.c_longlong, ctypes.c_longlong, _P, _P, _I, _P]),
    "lucid_guide_create": (_I, [_I, _I, ctypes.POINTER(_P)]),
    "lucid_guide_destroy": (None, [_P]),
    "lucid_guide_last_error": (ctypes.c_char_p, [_P]),
    "lucid_guide_num_params": (_I, []),
    "lucid_guide_get_params": (_I, [_P, _P, ctypes.c_size_t]),
    "lucid_guide_set_params": (_I, [_P, _P, ctypes.c_size_t]),
    "lucid_guide_forward": (_I, [_P, _P, _I, _P]),
    "lucid_guide_encode": (_I, [_P, _P, _P, _P, _I, _P]),
    "lucid_guide_gradient": (_I, [_P, _P, _I, _P]),
    "lucid_guide_train": (_I, [_P, _P, _I, ctypes.c_float]),
    "lucid_cuda_guide_enable": (_I, [_P, _I, _I]),
    "lucid_cuda_guide_steps": (_I, [_P]),
    "lucid_cuda_guide_config": (_I, [_P, _I, ctypes.c_float]),
    "lucid_cuda_guide_max_depth": (_I, [_P, _I]),
    "lucid_cuda_guide_params": (_I, [_P, _P, ctypes.c_size_t, _P]),
    "lucid_cuda_cancel": (_I, [_P]),
    "lucid_cuda_is_cancelled": (_I, [_P]),
    "lucid_cuda_reset_cancel": (_I, [_P]),
}

_lib = None


def load_library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("liblucid_cuda.so is not built (run blender-lucid-renderer_b200/build_ext.py); "
                               "the renderer has no CPU fallback")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class LucidError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lucid error {code}: {msg}")
        self.code = code


def inspect_scene(json_text: str, cap: int = 1 << 16):
    """Host-only parse: (counts[8], cdf, area, emission[n,3]) — no GPU needed."""
    lib = load_library()
    b = json_text.encode()
    counts = (ctypes.c_int * 8)()
    cdf = np.zeros(cap, np.float32)
    area = np.zeros(cap, np.float32)
    em = np.zeros((cap, 3), np.float32)
    n = lib.lucid_cuda_inspect_scene(b, len(b), counts, cdf.ctypes.data, area.ctypes.data, em.ctypes.data, cap)
    if n < 0:
        raise LucidError(n, "scene parse failed")
    n = min(n, cap)
    return list(counts), cdf[:n].copy(), area[:n].copy(), em[:n].copy()


class Context:
    """One renderer context on a CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.lucid_cuda_create(device, ctypes.byref(h))
        if rc != LUCID_OK:
            raise LucidError(rc, "create failed")
        self.h = h

    def close(self):
        if self.h:
            self.lib.lucid_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> int:
        if rc != LUCID_OK:
            raise LucidError(rc, self.lib.lucid_cuda_last_error(self.h).decode())
        return rc

    def _count(self, rc: int) -> int:
        """Calls that return a count on success and a negative status on failure."""
        if rc < 0:
            raise LucidError(rc, self.lib.lucid_cuda_last_error(self.h).decode())
        return rc

    def load_scene_json(self, text: str) -> None:
        b = text.encode()
        self._check(self.lib.lucid_cuda_load_scene_json(self.h, b, len(b)))

    def load_scene_arrays(self, arrays: dict) -> None:
        """Upload a scene given as arrays (lucid_scenes.scene_arrays)."""
        sd, keep = _scene_desc(arrays)
        self._check(self.lib.lucid_cuda_load_scene_arrays(self.h, ctypes.byref(sd)))
        del keep

    def set_launch_profile(self, profile: int) -> None:
        self._check(self.lib.lucid_cuda_set_launch_profile(self.h, profile))

    def update_scene(self, edits, check=True) -> int:
        """lucid_cuda_update_scene with scene_edits(edits)."""
        arr = scene_edits(edits)
        rc = self.lib.lucid_cuda_update_scene(self.h, ctypes.addressof(arr), len(edits))
        return self._check(rc) if check else rc

    def set_camera(self, *cam) -> None:
        self._check(self.lib.lucid_cuda_set_camera(self.h, *[float(c) for c in cam]))

    def set_algorithm(self, name: str) -> None:
        self._check(self.lib.lucid_cuda_set_algorithm(self.h, name.encode()))

    def set_wave_capacity(self, paths: int) -> None:
        self._check(self.lib.lucid_cuda_set_wave_capacity(self.h, int(paths)))

    def scene_stats(self):
        out = (ctypes.c_int * 8)()
        self._check(self.lib.lucid_cuda_scene_stats(self.h, out))
        return list(out)

    def device_info(self) -> str:
        buf = ctypes.create_string_buffer(256)
        self._check(self.lib.lucid_cuda_device_info(self.h, buf, 256))
        return buf.value.decode()

    def render(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
               tile_x=0, tile_y=0, records=False, profile=False, out=None, check=True):
        """Render into a host float32 RGBA array (tile_h, tile_w, 4).  Returns
        (image, records-or-None, status)."""
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        p = RenderParams(tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples, sample_offset, max_depth,
                         LUCID_RENDER_PROFILE if profile else 0)
        img = out if out is not None else np.zeros((tile_h, tile_w, 4), np.float32)
        recs = np.zeros(tile_w * tile_h * samples, RECORD_DTYPE) if records else None
        rc = self.lib.lucid_cuda_render(self.h, ctypes.byref(p), img.ctypes.data,
                                        recs.ctypes.data if recs is not None else None)
        if check:
            self._check(rc)
        return img, recs, rc

    def render_device(self, d_out_ptr: int, tile_w, tile_h, samples=1, sample_offset=0, max_depth=8,
                      profile=False):
        p = RenderParams(0, 0, tile_w, tile_h, tile_w, tile_h, samples, sample_offset, max_depth,
                         LUCID_RENDER_PROFILE if profile else 0)
        return self._check(self.lib.lucid_cuda_render_device(self.h, ctypes.byref(p), ctypes.c_void_p(d_out_ptr)))

    def render_noalloc(self, d_out_ptr: int, tile_w, tile_h, samples=1, sample_offset=0, max_depth=8,
                       check=True):
        """Render into caller-owned device memory without allocating (see
        lucid_cuda_render_noalloc in include/lucid_cuda.h for the limits)."""
        p = RenderParams(0, 0, tile_w, tile_h, tile_w, tile_h, samples, sample_offset, max_depth, 0)
        rc = self.lib.lucid_cuda_render_noalloc(self.h, ctypes.byref(p), ctypes.c_void_p(d_out_ptr))
        return self._check(rc) if check else rc

    def set_combining(self, on: bool) -> None:
        """lucid_cuda_set_combining: take part in (or stay out of) the
        device's combining of concurrent small renders."""
        self._check(self.lib.lucid_cuda_set_combining(self.h, int(bool(on))))

    def render_batch(self, jobs, algorithm: str = "mis", check=True):
        """lucid_cuda_render_batch: `jobs` is a list of dicts with `scene` (a
        Context with a loaded scene), `camera` (10 floats), `width`, `height`
        and optionally `samples`, `sample_offset`, `max_depth` (8), `tile_x`,
        `tile_y`, `full_w`, `full_h` (a tile of a larger image).  Returns
        ([image per job], status); each image is (height, width, 4) float32."""
        arr = (BatchJob * len(jobs))()
        imgs = []
        for k, j in enumerate(jobs):
            w, h = int(j["width"]), int(j["height"])
            img = np.zeros((h, w, 4), np.float32)
            imgs.append(img)
            arr[k].scene = j["scene"].h
            arr[k].camera = (ctypes.c_float * 10)(*[float(c) for c in j["camera"]])
            arr[k].params = RenderParams(int(j.get("tile_x", 0)), int(j.get("tile_y", 0)), w, h,
                                         int(j.get("full_w", w)), int(j.get("full_h", h)), int(j.get("samples", 1)),
                                         int(j.get("sample_offset", 0)), int(j.get("max_depth", 8)), 0)
            arr[k].out_rgba = img.ctypes.data
        rc = self.lib.lucid_cuda_render_batch(self.h, ctypes.addressof(arr), len(jobs), algorithm.encode())
        if check:
            self._check(rc)
        return imgs, rc

    def render_debug(self, mode: str, tile_w, tile_h, full_w=None, full_h=None, tile_x=0, tile_y=0):
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        img = np.zeros((tile_h, tile_w, 4), np.float32)
        self._check(self.lib.lucid_cuda_render_debug(self.h, tile_x, tile_y, tile_w, tile_h, full_w, full_h,
                                                     mode.encode(), img.ctypes.data))
        return img

    def stats(self) -> dict:
        s = RenderStats()
        self._check(self.lib.lucid_cuda_get_stats(self.h, ctypes.byref(s)))
        kinds = {}
        for k in range(s.num_kinds):
            ks = s.kinds[k]
            kinds[ks.name.decode()] = {"launches": ks.launches, "total_ms": ks.total_ms,
                                       "algo_bytes": ks.algo_bytes, "units": ks.units}
        return {"total_ms": s.total_ms, "paths": s.paths, "segments": s.segments, "shadow_rays": s.shadow_rays,
                "waves": s.waves, "kernels": kinds}

    # progressive accumulator (viewport)
    def async_start(self, w, h, max_depth=8):
        self._check(self.lib.lucid_cuda_async_start(self.h, w, h, max_depth))
        self._async_shape = (h, w)

    def async_poll(self):
        h, w = getattr(self, "_async_shape", (0, 0))
        n = ctypes.c_int(0)
        img = np.zeros((h, w, 4), np.float32)
        self._check(self.lib.lucid_cuda_async_poll(self.h, ctypes.byref(n), img.ctypes.data, img.size))
        return n.value, (img if n.value > 0 else None)

    def async_revision(self) -> int:
        return self.lib.lucid_cuda_async_revision(self.h)

    def async_reset(self, w, h, max_depth=8):
        self._check(self.lib.lucid_cuda_async_reset(self.h, w, h, max_depth))

    def async_stop(self):
        self._check(self.lib.lucid_cuda_async_stop(self.h))

    def async_running(self) -> bool:
        return self.lib.lucid_cuda_async_running(self.h) == 1

    def cancel(self):
        self.lib.lucid_cuda_cancel(self.h)

    def is_cancelled(self) -> bool:
        return self.lib.lucid_cuda_is_cancelled(self.h) == 1

    def render_f64(self, tile_w, tile_h, full_w=None, full_h=None, samples=1, sample_offset=0, max_depth=8,
                   tile_x=0, tile_y=0):
        """Per-pixel FP64 sum of the samples' FP32 radiance (a converged reference
        is this divided by samples)."""
        full_w = tile_w if full_w is None else full_w
        full_h = tile_h if full_h is None else full_h
        p = RenderParams(tile_x, tile_y, tile_w, tile_h, full_w, full_h, samples, sample_offset, max_depth, 0)
        img = np.zeros((tile_h, tile_w, 4), np.float64)
        self._check(self.lib.lucid_cuda_render_f64(self.h, ctypes.byref(p), img.ctypes.data))
        return img

    def guide_enable(self, on: bool = True, seed: int = 1):
        self._check(self.lib.lucid_cuda_guide_enable(self.h, int(on), seed))

    def guide_config(self, steps_per_wave: int = 2, lr: float = 1e-2):
        self._check(self.lib.lucid_cuda_guide_config(self.h, steps_per_wave, ctypes.c_float(lr)))

    def guide_max_depth(self, max_depth: int = 1):
        self._check(self.lib.lucid_cuda_guide_max_depth(self.h, max_depth))

    def guide_params(self):
        """(FP32 weights, scene box (lo, hi)) of this context's guide network."""
        n = self.lib.lucid_guide_num_params()
        w = np.zeros(n, np.float32)
        box = np.zeros(6, np.float32)
        self._count(self.lib.lucid_cuda_guide_params(self.h, w.ctypes.data, w.size, box.ctypes.data))
        return w, (box[:3].copy(), box[3:].copy())

    def guide_steps(self) -> int:
        return self._count(self.lib.lucid_cuda_guide_steps(self.h))

    # ---- path diagnostics ----
    def diag_enable(self, subsample=2, record_capacity=0):
        cfg = DiagConfig(subsample, 16, 4, 16, 0.001, 3.0, record_capacity)
        self._check(self.lib.lucid_cuda_diag_enable(self.h, ctypes.byref(cfg)))

    def diag_disable(self):
        self._check(self.lib.lucid_cuda_diag_disable(self.h))

    def diag_enabled(self) -> bool:
        return self.lib.lucid_cuda_diag_enabled(self.h) == 1

    def diag_clear(self):
        self._check(self.lib.lucid_cuda_diag_clear(self.h))

    def diag_stats(self) -> list:
        out = np.zeros(5, np.uint64)
        self._check(self.lib.lucid_cuda_diag_stats(self.h, out.ctypes.data))
        return out.tolist()

    def diag_pixel(self, x, y, sort_by_mean=False, cap=32):
        info = np.zeros(1, DIAG_PIXEL_DTYPE)
        groups = np.zeros(cap, DIAG_GROUP_DTYPE)
        n = self._count(self.lib.lucid_cuda_diag_pixel(self.h, x, y, int(sort_by_mean), info.ctypes.data,
                                                       groups.ctypes.data, cap))
        return info[0], groups[:n]

    def diag_variance_map(self, w, h):
        out = np.zeros(w * h, np.float32)
        n = self._count(self.lib.lucid_cuda_diag_variance_map(self.h, out.ctypes.data, out.size))
        return out[:n]

    def diag_coarse_stats(self) -> list:
        out = (DiagCoarse * 8)()
        self._count(self.lib.lucid_cuda_diag_coarse_stats(self.h, ctypes.addressof(out)))
        return [(c.type_id, c.name.decode(), c.sample_count, c.mean_luminance, c.variance_luminance,
                 tuple(c.mean_rgb), tuple(c.variance_rgb)) for c in out]

    def diag_suggestions(self) -> list:
        out = (DiagSuggestion * 8)()
        n = self._count(self.lib.lucid_cuda_diag_suggestions(self.h, ctypes.addressof(out), 8))
        return [(s.category.decode(), s.severity.decode(), s.message.decode(), s.action.decode())
                for s in out[:min(n, 8)]]

    def diag_export_binary(self) -> bytes:
        n = self._count(self.lib.lucid_cuda_diag_export_binary(self.h, None, 0))
        buf = ctypes.create_string_buffer(max(n, 1))
        self.lib.lucid_cuda_diag_export_binary(self.h, buf, n)
        return buf.raw[:n]

    def diag_metadata_json(self) -> str:
        n = self._count(self.lib.lucid_cuda_diag_metadata_json(self.h, None, 0))
        buf = ctypes.create_string_buffer(n + 1)
        self.lib.lucid_cuda_diag_metadata_json(self.h, buf, n + 1)
        return buf.value.decode()

    def diag_top_groups(self, n, by_mean=False):
        groups = np.zeros(max(n, 1), DIAG_GROUP_DTYPE)
        xy = np.zeros((max(n, 1), 2), np.int32)
        m = self._count(self.lib.lucid_cuda_diag_top_groups(self.h, n, int(by_mean), groups.ctypes.data,
                                                            xy.ctypes.data, groups.size))
        return groups[:m], xy[:m]


def scene_digest(json_text: str | None = None, arrays: dict | None = None) -> int:
    """Host-only digest of the scene either form would upload (no GPU)."""
    lib = load_library()
    out = ctypes.c_uint64(0)
    if json_text is not None:
        b = json_text.encode()
        rc = lib.lucid_scene_digest(b, len(b), None, ctypes.byref(out))
    else:
        sd, keep = _scene_desc(arrays)
        rc = lib.lucid_scene_digest(None, 0, ctypes.byref(sd), ctypes.byref(out))
        del keep
    if rc != LUCID_OK:
        raise LucidError(rc, "invalid scene")
    return out.value


def batch_plan(max_paths: int, room_bytes: int, jobs, cancelled=None) -> list:
    """The server's batching policy run on the host (no GPU): `jobs` is a
    list of dicts (scene, width, height, samples, max_depth, algorithm,
    interactive, guided), the first taken from the head of the queue, the
    rest waiting behind it; returns the 0/1 membership of each in the
    head's batch."""
    lib = load_library()
    arr = (JobDesc * len(jobs))()
    for k, j in enumerate(jobs):
        arr[k] = JobDesc(int(j.get("scene", 0)), (ctypes.c_float * 10)(), j.get("algorithm", "mis").encode(),
                         int(j["width"]), int(j["height"]), int(j["samples"]), int(j.get("max_depth", 8)),
                         int(j.get("interactive", 0)), int(j.get("guided", 0)), 1)
    canc = (ctypes.c_int * len(jobs))(*[int(c) for c in (cancelled or [0] * len(jobs))])
    member = (ctypes.c_int * len(jobs))()
    rc = lib.lucid_batch_plan(int(max_paths), int(room_bytes), ctypes.addressof(arr), ctypes.addressof(canc),
                              len(jobs), ctypes.addressof(member))
    if rc < 0:
        raise LucidError(rc, "batch_plan failed")
    return list(member)


def batch_bytes(pixels: int, paths: int) -> int:
    """Device bytes of a batch of `pixels` image pixels and `paths` paths in one wave."""
    return paths * 178 + pixels * 32 + (2 << 20)


def admission_plan(budget: int, reserved: int, slots: int, job_bytes) -> list:
    """The server's admission policy run on the host (no GPU): the start order
    of each job when jobs finish in start order, or -1 when it is refused."""
    lib = load_library()
    b = np.asarray(job_bytes, np.int64)
    out = np.zeros(len(b), np.int32)
    rc = lib.lucid_admission_plan(int(budget), int(reserved), int(slots), b.ctypes.data, len(b), out.ctypes.data)
    if rc != LUCID_OK:
        raise LucidError(rc, "admission plan")
    return out.tolist()


def combine_stats(device: int = 0):
    """(batches, calls) the device's combiner of concurrent small renders has run."""
    lib = load_library()
    b, c = ctypes.c_longlong(), ctypes.c_longlong()
    lib.lucid_cuda_combine_stats(device, ctypes.byref(b), ctypes.byref(c))
    return b.value, c.value


class Server:
    """Several progressive render jobs on one device (the request loop)."""

    def __init__(self, device: int = 0, slots: int = 4, budget_bytes: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.lucid_server_create(device, slots, budget_bytes, ctypes.byref(h))
        if rc != LUCID_OK:
            raise LucidError(rc, "server create failed")
        self.h = h
        self._sizes = {}

    def close(self):
        if self.h:
            self.lib.lucid_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc):
        raise LucidError(rc, self.lib.lucid_server_last_error(self.h).decode())

    def add_scene(self, json_text: str) -> int:
        b = json_text.encode()
        sid = ctypes.c_int()
        rc = self.lib.lucid_server_add_scene(self.h, b, len(b), ctypes.byref(sid))
        if rc != LUCID_OK:
            self._err(rc)
        return sid.value

    def add_scene_arrays(self, arrays: dict) -> int:
        sd, keep = _scene_desc(arrays)
        sid = ctypes.c_int()
        rc = self.lib.lucid_server_add_scene_arrays(self.h, ctypes.byref(sd), ctypes.byref(sid))
        del keep
        if rc != LUCID_OK:
            self._err(rc)
        return sid.value

    def update_scene(self, scene: int, edits, check=True) -> int:
        """lucid_server_update_scene: jobs submitted afterwards see the edits."""
        arr = scene_edits(edits)
        rc = self.lib.lucid_server_update_scene(self.h, scene, ctypes.addressof(arr), len(edits))
        if rc != LUCID_OK and check:
            self._err(rc)
        return rc

    def submit(self, scene: int, camera, width: int, height: int, samples: int, max_depth: int = 8,
               algorithm: str = "mis", interactive: bool = False, check: bool = True, guided: bool = False,
               guide_seed: int = 1):
        d = JobDesc(scene, (ctypes.c_float * 10)(*[float(c) for c in camera]), algorithm.encode(), width, height,
                    samples, max_depth, int(interactive), int(guided), guide_seed)
        jid = ctypes.c_int()
        rc = self.lib.lucid_server_submit(self.h, ctypes.byref(d), ctypes.byref(jid))
        self._sizes[jid.value] = (height, width)
        if rc != LUCID_OK and check:
            self._err(rc)
        return jid.value

    def state(self, job: int):
        n = ctypes.c_int()
        st = self.lib.lucid_server_job_state(self.h, job, ctypes.byref(n))
        return st, n.value

    def wait(self, job: int, timeout_ms: int = -1) -> int:
        return self.lib.lucid_server_wait(self.h, job, timeout_ms)

    def result(self, job: int) -> np.ndarray:
        h, w = self._sizes[job]
        img = np.zeros((h, w, 4), np.float32)
        rc = self.lib.lucid_server_result(self.h, job, img.ctypes.data, img.size)
        if rc != LUCID_OK:
            self._err(rc)
        return img

    def cancel(self, job: int):
        self.lib.lucid_server_cancel(self.h, job)

    def set_batching(self, max_paths: int) -> None:
        """lucid_server_set_batching: batches of at most max_paths paths (0: off)."""
        rc = self.lib.lucid_server_set_batching(self.h, int(max_paths))
        if rc != LUCID_OK:
            self._err(rc)

    def stats(self) -> dict:
        st = ServerStats()
        rc = self.lib.lucid_server_stats(self.h, ctypes.byref(st))
        if rc != LUCID_OK:
            self._err(rc)
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}


class DiagFilm:
    """A standalone DiagnosticFilm (lucid_diag_film_*, host only: no GPU)."""

    def __init__(self, width: int, height: int, subsample: int = 2, max_groups: int = 16, max_outliers: int = 4,
                 max_depth: int = 16, variance_threshold: float = 0.001, outlier_threshold: float = 3.0):
        self.lib = load_library()
        cfg = DiagConfig(subsample, max_groups, max_outliers, max_depth, variance_threshold, outlier_threshold, 0)
        h = ctypes.c_void_p()
        rc = self.lib.lucid_diag_film_create(width, height, ctypes.byref(cfg), ctypes.byref(h))
        if rc != LUCID_OK:
            raise LucidError(rc, "lucid_diag_film_create failed")
        self.h = h

    def close(self):
        if self.h:
            self.lib.lucid_diag_film_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def record_path(self, x: int, y: int, trace: PathTrace):
        rc = self.lib.lucid_diag_film_record_path(self.h, x, y, ctypes.byref(trace))
        if rc != LUCID_OK:
            raise LucidError(rc, "record_path failed")

    def clear(self):
        self.lib.lucid_diag_film_clear(self.h)

    def info(self) -> list:
        v = (ctypes.c_longlong * 5)()
        self.lib.lucid_diag_film_info(self.h, v)
        return list(v)

    def pixel(self, x, y, sort_by_mean=False, cap=32):
        info = np.zeros(1, DIAG_PIXEL_DTYPE)
        groups = np.zeros(cap, DIAG_GROUP_DTYPE)
        n = self.lib.lucid_diag_film_pixel(self.h, x, y, int(sort_by_mean), info.ctypes.data, groups.ctypes.data, cap)
        if n < 0:
            raise LucidError(n, "pixel query failed")
        return info[0], groups[:n]

