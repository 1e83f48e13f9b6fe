"""Converged references and the relMSE error metric.

A reference image is the per-pixel mean of many samples (4096 by default)
accumulated in FP64 on the GPU (`lucid_cuda_render_f64`); relMSE is the mean
over pixels and channels of (x - ref)^2 / (ref^2 + eps) with eps = 1e-2.

Command line (writes an .npy of shape (h, w, 3), float64, Y-flipped like
render_tile):

    python lucid_quality.py scene.json --camera px py pz dx dy dz ux uy uz fov \
        --width 256 --height 256 --spp 4096 --depth 8 --algorithm mis --out ref.npy
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

REL_EPS = 1e-2
REFERENCE_SPP = 4096


def relmse(img: np.ndarray, ref: np.ndarray, eps: float = REL_EPS) -> float:
    """Relative MSE of an image against a reference (RGB; extra channels are
    ignored): mean over pixels and channels of (x - ref)^2 / (ref^2 + eps)."""
    x = np.asarray(img, dtype=np.float64)[..., :3]
    r = np.asarray(ref, dtype=np.float64)[..., :3]
    if x.shape != r.shape:
        raise ValueError(f"shape mismatch {x.shape} vs {r.shape}")
    return float(np.mean((x - r) ** 2 / (r * r + eps)))


def mean_image(sum_rgba: np.ndarray, samples: int) -> np.ndarray:
    """Per-pixel mean RGB from a render's per-pixel sum over its samples."""
    return np.asarray(sum_rgba, dtype=np.float64)[..., :3] / float(samples)


def render_reference(ctx, width: int, height: int, spp: int = REFERENCE_SPP, max_depth: int = 8,
                     tile=None, sample_offset: int = 0) -> np.ndarray:
    """FP64 reference (per-pixel mean RGB) rendered on the GPU through `ctx`
    (a lucid_capi.Context with scene, camera and algorithm set).  One call:
    the engine splits the samples into waves and sums every sample's FP32
    radiance in FP64 in sample order."""
    tx, ty, tw, th = tile if tile else (0, 0, width, height)
    s = ctx.render_f64(tw, th, width, height, spp, sample_offset, max_depth, tile_x=tx, tile_y=ty)
    return mean_image(s, spp)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("scene")
    ap.add_argument("--camera", type=float, nargs=10, required=True)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--height", type=int, default=256)
    ap.add_argument("--spp", type=int, default=REFERENCE_SPP)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--algorithm", default="mis")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", required=True)
    args = ap.parse_args(argv)
    import lucid_capi
    ctx = lucid_capi.Context(args.device)
    with open(args.scene) as f:
        ctx.load_scene_json(f.read())
    ctx.set_camera(*args.camera)
    ctx.set_algorithm(args.algorithm)
    ref = render_reference(ctx, args.width, args.height, args.spp, args.depth)
    np.save(args.out, ref)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
