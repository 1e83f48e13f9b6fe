"""The C ABI library loads on a machine without a GPU and exports every
function include/lucid_cuda.h declares; the ctypes binding covers them all."""
import ctypes
import os
import re

import lucid_capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(REPO, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(REPO, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(lucid_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(lucid_capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names <= set(lucid_capi.SIGNATURES), names - set(lucid_capi.SIGNATURES)


def test_context_without_gpu_reports_errors_not_crashes():
    ctx = lucid_capi.Context(0)   # creating a context touches no device
    img, _, rc = ctx.render(4, 4, check=False)
    assert rc == lucid_capi.LUCID_ERR_NO_SCENE
    assert not img.any()
    assert ctx.lib.lucid_cuda_render(None, None, None, None) == lucid_capi.LUCID_ERR_INVALID
    ctx.cancel()
    assert ctx.is_cancelled()
    ctx.close()


def test_pybind_module_surface():
    import lucidrenderer as lr
    r = lr.Renderer()
    for m in ("cancel", "is_cancelled", "reset_cancel", "load_scene_json", "set_camera", "set_algorithm",
              "render_tile", "render_tile_gpu", "render_tile_numpy", "render_debug", "render_debug_gpu",
              "set_object_names", "get_object_name", "object_path_string", "is_scene_loaded", "is_camera_set",
              "get_algorithm", "get_mesh_count"):
        assert hasattr(r, m), m
    assert r.get_algorithm() == "nee"
    assert lr.cuda_enabled and not lr.dawn_enabled
    assert r.get_object_name(-1) == "Environment" and r.get_object_name(7) == "Object_7"
    r.set_object_names(["Floor", "Lamp"])
    assert r.object_path_string([0, -1]) == "Environment(?) → Floor → Camera"
    assert r.load_scene_json("{broken") is False
    # no scene / camera: a zero buffer, like the reference (pybind_renderer.hpp:200-203)
    px = r.render_tile(0, 0, 4, 4, 4, 4)
    assert len(px) == 64 and not any(px)
