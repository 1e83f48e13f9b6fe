"""Generate the golden per-sample fixtures from the CPU oracle.

The reference's tests pin no pixel or RNG values, so these fixtures are made
by the oracle (the CPU restatement of the reference integrators, shared
deterministic math, canonical tie rule) and committed; the GPU tests compare
the CUDA tracer against them and the CPU tests check the oracle still
reproduces them.

    python tests/golden/make_golden.py
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

# name -> (scene, algorithm, width, height, spp, depth, sample_offset)
CASES = {
    "cornell_mis": ("cornell", "mis", 16, 16, 4, 8, 0),
    "cornell_nee": ("cornell", "nee", 12, 12, 2, 8, 5),
    "all_lights_volume_mis": ("all_lights", "volume_mis", 16, 12, 2, 8, 1),
    "mirror_mis": ("mirror", "mis", 12, 12, 2, 6, 0),
}


def render_case(name, workdir):
    from parity_util import render_oracle, scene_and_camera
    scene, algo, w, h, spp, depth, off = CASES[name]
    sc, cam = scene_and_camera(scene, workdir)
    img, recs = render_oracle(sc, cam, algo, w, h, spp, depth, offset=off)
    return img, recs


def main():
    with tempfile.TemporaryDirectory() as wd:
        for name in CASES:
            img, recs = render_case(name, wd)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), image=img, records=recs)
            print(name, img.shape, len(recs))


if __name__ == "__main__":
    main()
