"""Multi-process path on CPU (gloo, world size 2).

A render is sharded across ranks by sample range: rank r renders the same
tile with sample_offset = r * S and the films are summed with one
all_reduce.  Because seeds are (x, y, offset + s), the sharded sum equals the
sequential renders of the two sample ranges exactly.  The CPU oracle stands
in for the device tracer here; the sharding logic is the one bench.py uses
(weak scaling, one reduction at the end of a job)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
W, H, S = 12, 10, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _render(offset):
    import sys
    sys.path[:0] = [os.path.join(REPO, "blender-lucid-renderer_b200"), os.path.join(REPO, "oracle")]
    import lucid_scenes as ls
    from oracle_ctypes import Oracle
    sc, cam = ls.cornell_box()
    o = Oracle()
    assert o.load_scene_json(ls.to_json(sc))
    o.set_camera(*cam)
    o.set_algorithm("mis")
    img, _, rc = o.render(W, H, W, H, S, offset, 8)
    assert rc == 0
    return img


def _worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    film = torch.from_numpy(_render(rank * S).copy())
    dist.all_reduce(film, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.save(out_path, film.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_sample_range_sharding_matches_sequential(tmp_path):
    out = str(tmp_path / "film.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    got = np.load(out)
    want = _render(0) + _render(S)
    # alpha is summed too (2 ranks); colour channels must match exactly
    assert np.array_equal(got[..., :3], want[..., :3])
