"""Online path guiding in the renderer (GPU): the guided estimator is
unbiased (its image mean matches a plain FP64 reference within 4 standard
errors) and the network it trains lowers the error at equal samples on the
hard-indirect room (light reaches it only through a 0.5 m door gap)."""
from __future__ import annotations

import numpy as np
import pytest

import lucid_quality as lq
import lucid_scenes as ls

pytestmark = pytest.mark.gpu


def _ctx(scene, cam):
    import lucid_capi
    c = lucid_capi.Context(0)
    c.load_scene_json(ls.to_json(scene))
    c.set_camera(*cam)
    c.set_algorithm("mis")
    return c


@pytest.mark.parametrize("guided_depth", [1, 8])
def test_guided_render_is_unbiased(guided_depth):
    scene, cam = ls.cornell_box()
    ctx = _ctx(scene, cam)
    W = H = 64
    ref = lq.render_reference(ctx, W, H, spp=4096, max_depth=8, sample_offset=1 << 20)
    ctx.guide_max_depth(guided_depth)
    ctx.guide_enable(True, 5)
    means = []
    for k in range(48):
        img, _, _ = ctx.render(W, H, W, H, 8, 8 * k, 8)
        means.append(lq.mean_image(img, 8).mean())
    assert ctx.guide_steps() > 0
    means = np.array(means)
    se = means.std(ddof=1) / np.sqrt(len(means))
    assert abs(means.mean() - ref.mean()) < 4 * se + 1e-4 * ref.mean()
    ctx.guide_enable(False, 0)
    ctx.close()


def test_trained_guide_lowers_error_at_equal_samples():
    scene, cam = ls.hard_indirect_scene()
    ctx = _ctx(scene, cam)
    W, H, spp, calls = 320, 180, 4, 160
    ref = lq.render_reference(ctx, W, H, spp=4096, max_depth=8, sample_offset=1 << 20)
    errs = {}
    for guided in (False, True):
        if guided:
            ctx.guide_config(4, 1e-2)
            ctx.guide_max_depth(8)
            ctx.guide_enable(True, 1)
        else:
            ctx.guide_enable(False, 0)
        acc = np.zeros((H, W, 4))
        for k in range(calls):
            acc += ctx.render(W, H, W, H, spp, spp * k, 8)[0]
        errs[guided] = lq.relmse(lq.mean_image(acc, calls * spp), ref)
    assert errs[True] < 0.95 * errs[False], errs
    ctx.close()
