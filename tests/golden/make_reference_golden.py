"""Generate golden images from the Lucid reference itself.

The reference's own CPU render path (PyRenderer::render_tile / render_debug,
LucidRenderer/cpp_renderer/include/pybind_renderer.hpp) is built here from its
unmodified sources against the project-written mp-units shim
(`make -C oracle ref`, oracle/_ref/libref_check.so) and run on small seeded
scenes; the images are committed as tests/golden/ref_*.npz.  The CPU tests
check that the oracle, run the way that build runs (libm, the reference's
traversal and tie order, call-argument draws right to left), reproduces them
bit for bit, also where the reference sources and library are absent.

    make -C oracle ref && python tests/golden/make_reference_golden.py
"""
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "blender-lucid-renderer_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import numpy as np  # noqa: E402

# name -> (scene, algorithm or "debug:<mode>", width, height, spp, depth, sample_offset)
REF_CASES = {
    "ref_cornell_mis": ("cornell", "mis", 32, 32, 4, 8, 0),
    "ref_cornell_simple": ("cornell", "simple", 16, 16, 2, 8, 2),
    "ref_all_lights_volume_mis": ("all_lights", "volume_mis", 24, 18, 2, 8, 1),
    "ref_all_lights_nee": ("all_lights_novol", "nee", 24, 18, 2, 8, 0),
    "ref_textured_mis": ("textured", "mis", 24, 18, 2, 8, 0),
    "ref_hard_indirect_mis": ("hard_indirect", "mis", 24, 16, 2, 8, 0),
    "ref_procedural_small_volume_mis": ("procedural_small", "volume_mis", 24, 16, 2, 12, 3),
    "ref_all_lights_debug_normal": ("all_lights", "debug:normal", 24, 18, 1, 1, 0),
    "ref_textured_debug_albedo": ("textured", "debug:albedo", 24, 18, 1, 1, 0),
}


def render_reference(name, workdir):
    import lucid_scenes as ls
    import ref_ctypes
    from parity_util import scene_and_camera
    scene, algo, w, h, spp, depth, off = REF_CASES[name]
    sc, cam = scene_and_camera(scene, workdir)
    r = ref_ctypes.ReferenceRenderer()
    assert r.load_scene_json(ls.to_json(sc))
    r.set_camera(*cam)
    if algo.startswith("debug:"):
        return r.render_debug(algo.split(":", 1)[1], w, h)
    r.set_algorithm(algo)
    return r.render(w, h, w, h, spp, off, depth)


def main():
    with tempfile.TemporaryDirectory() as wd:
        for name in REF_CASES:
            img = render_reference(name, wd)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), image=img)
            print(name, img.shape, float(img[..., :3].mean()))


if __name__ == "__main__":
    main()
