"""GPU test of lucid_cuda_render_noalloc, the entry point for callers that
cannot allocate device memory while rendering (a host whose device memory
belongs to another allocator, or a draw-callback thread that must not call
cudaMalloc/cudaFree because they can synchronise the device).  It must give
the same image as lucid_cuda_render_device on consecutive calls, although the
fixed scratch array keeps the previous call's contents.  This file is
collected last so a failure here comes after every other test has run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H, SPP, DEPTH = 64, 48, 4, 8


@pytest.fixture(scope="module")
def scene_ctx():
    import torch
    import lucid_capi
    import lucid_scenes as ls
    ctx = lucid_capi.Context(0)
    sc, cam = ls.cornell_box()
    ctx.load_scene_json(ls.to_json(sc))
    ctx.set_camera(*cam)
    ctx.set_algorithm("mis")
    yield ctx, torch
    ctx.close()


def test_noalloc_matches_render_device_twice(scene_ctx):
    ctx, torch = scene_ctx
    ref = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ctx.render_device(ref.data_ptr(), W, H, SPP, 0, DEPTH)
    torch.cuda.synchronize()
    want = ref.cpu().numpy()
    assert want[..., :3].sum() > 0
    for call in range(2):
        out = torch.full((H, W, 4), -1.0, dtype=torch.float32, device="cuda")
        ctx.render_noalloc(out.data_ptr(), W, H, SPP, 0, DEPTH)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-4, atol=1e-5, err_msg=f"call {call}")


def test_noalloc_rejects_requests_beyond_its_scratch(scene_ctx):
    ctx, torch = scene_ctx
    import lucid_capi
    out = torch.zeros((300, 300, 4), dtype=torch.float32, device="cuda")
    rc = ctx.render_noalloc(out.data_ptr(), 300, 300, 1, 0, DEPTH, check=False)   # 90,000 px > 65,536
    assert rc == lucid_capi.LUCID_ERR_INVALID
    assert "limit" in ctx.lib.lucid_cuda_last_error(ctx.h).decode()
    rc = ctx.render_noalloc(out.data_ptr(), 16, 16, 1, 0, 65, check=False)         # depth > 64
    assert rc == lucid_capi.LUCID_ERR_INVALID
