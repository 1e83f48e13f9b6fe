"""GPU tests of lucid_cuda_render_noalloc, the entry point for callers that
cannot allocate device memory while rendering (a host whose device memory
belongs to another allocator, or a draw-callback thread that must not call
cudaMalloc/cudaFree because they can synchronise the device).  It must give
the same image as lucid_cuda_render_device on consecutive calls, although the
fixed scratch array keeps the previous call's contents: single-wave tiles,
tiles that take several waves of the fixed path pool (the per-wave counters
are cleared, the film sums across waves, the sample offset of each wave moves
on), an odd-sized tile whose samples do not divide into equal waves, and the
nee / volume_mis integrators.  This file is collected last so a failure here
comes after every other test has run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEPTH = 8


@pytest.fixture(scope="module")
def torch_mod():
    import torch
    return torch


def _ctx(scene_fn, algo, tmp_path_factory=None):
    import lucid_capi
    import lucid_scenes as ls
    ctx = lucid_capi.Context(0)
    if scene_fn == "all_lights":
        d = tmp_path_factory.mktemp("noalloc")
        sc, cam = ls.all_lights_scene(str(d), with_volume=True)
    else:
        sc, cam = ls.cornell_box()
    ctx.load_scene_json(ls.to_json(sc))
    ctx.set_camera(*cam)
    ctx.set_algorithm(algo)
    return ctx


def _check_twice(ctx, torch, w, h, spp, offset=0):
    ref = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    ctx.render_device(ref.data_ptr(), w, h, spp, offset, DEPTH)
    torch.cuda.synchronize()
    want = ref.cpu().numpy()
    assert want[..., :3].sum() > 0
    for call in range(2):
        out = torch.full((h, w, 4), -1.0, dtype=torch.float32, device="cuda")
        ctx.render_noalloc(out.data_ptr(), w, h, spp, offset, DEPTH)
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-4, atol=1e-5,
                                   err_msg=f"{w}x{h} {spp} spp, call {call}")


@pytest.mark.parametrize("w,h,spp,offset", [
    (64, 48, 4, 0),        # one wave
    (256, 256, 4, 0),      # four waves of 65,536 paths
    (203, 151, 5, 7),      # 30,653 px: waves of 2, 2 and 1 samples, non-zero sample offset
])
def test_noalloc_matches_render_device_cornell_mis(torch_mod, w, h, spp, offset):
    ctx = _ctx("cornell", "mis")
    try:
        _check_twice(ctx, torch_mod, w, h, spp, offset)
    finally:
        ctx.close()


@pytest.mark.parametrize("algo", ["nee", "volume_mis"])
def test_noalloc_matches_render_device_other_integrators(torch_mod, tmp_path_factory, algo):
    ctx = _ctx("all_lights", algo, tmp_path_factory)
    try:
        _check_twice(ctx, torch_mod, 203, 151, 5, 3)   # several uneven waves
    finally:
        ctx.close()


def test_noalloc_matches_the_oracle(torch_mod):
    """The no-allocation render checked against the CPU oracle directly
    (Cornell, mis, two waves' worth of samples at 96x80)."""
    import lucid_scenes as ls
    from parity_util import render_oracle
    sc, cam = ls.cornell_box()
    w, h, spp = 96, 80, 12
    ctx = _ctx("cornell", "mis")
    out = torch_mod.full((h, w, 4), -1.0, dtype=torch_mod.float32, device="cuda")
    ctx.render_noalloc(out.data_ptr(), w, h, spp, 0, DEPTH)
    torch_mod.cuda.synchronize()
    ctx.close()
    want, _ = render_oracle(sc, cam, "mis", w, h, spp, DEPTH)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-6, atol=1e-7)


def test_noalloc_rejects_requests_beyond_its_scratch(torch_mod):
    import lucid_capi
    torch = torch_mod
    ctx = _ctx("cornell", "mis")
    try:
        out = torch.zeros((300, 300, 4), dtype=torch.float32, device="cuda")
        rc = ctx.render_noalloc(out.data_ptr(), 300, 300, 1, 0, DEPTH, check=False)   # 90,000 px > 65,536
        assert rc == lucid_capi.LUCID_ERR_INVALID
        assert "limit" in ctx.lib.lucid_cuda_last_error(ctx.h).decode()
        rc = ctx.render_noalloc(out.data_ptr(), 16, 16, 1, 0, 65, check=False)         # depth > 64
        assert rc == lucid_capi.LUCID_ERR_INVALID
    finally:
        ctx.close()


def test_noalloc_refuses_guiding_and_diagnostics(torch_mod):
    """Path guiding and path diagnostics keep buffers this entry point cannot
    allocate; it refuses rather than render a different image."""
    import lucid_capi
    torch = torch_mod
    ctx = _ctx("cornell", "mis")
    try:
        out = torch.zeros((32, 32, 4), dtype=torch.float32, device="cuda")
        ctx.guide_enable(True)
        rc = ctx.render_noalloc(out.data_ptr(), 32, 32, 1, 0, DEPTH, check=False)
        assert rc == lucid_capi.LUCID_ERR_INVALID
        assert "guiding" in ctx.lib.lucid_cuda_last_error(ctx.h).decode()
        ctx.guide_enable(False)
        ctx.diag_enable(subsample=1)
        rc = ctx.render_noalloc(out.data_ptr(), 32, 32, 1, 0, DEPTH, check=False)
        assert rc == lucid_capi.LUCID_ERR_INVALID
        assert "diagnostics" in ctx.lib.lucid_cuda_last_error(ctx.h).decode()
        ctx.diag_disable()
        ctx.render_noalloc(out.data_ptr(), 32, 32, 1, 0, DEPTH)   # both off: renders again
        torch.cuda.synchronize()
        assert float(out[..., :3].sum()) > 0
    finally:
        ctx.close()
