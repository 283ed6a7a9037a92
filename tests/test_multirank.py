"""Host-side sharding used by `bench.py --gpus N`: every rank renders its own
pass range; summing the ranks' accumulation buffers equals one render of all
passes.  Runs two `gloo` ranks on the CPU with the FP64 oracle standing in
for the device render."""

import os
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out_path):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "embree-benchmark-protoray_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    import oracle
    import scenes
    mesh, view = scenes.small_scene()
    O = oracle.Oracle()
    s = O.scene(mesh.positions, mesh.indices)
    W, H, spp, depth = 16, 12, 2, 3
    pass0, npass = bench.rank_pass_range(rank, world, spp)
    acc, rays = s.render(O.camera(view, W, H), W, H, pass0, npass, depth, nthreads=1)
    t = torch.from_numpy(acc)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    r = torch.tensor([float(rays)], dtype=torch.float64)
    dist.all_reduce(r, op=dist.ReduceOp.SUM)
    if rank == 0:
        np.save(out_path, np.concatenate([t.numpy().ravel(), r.numpy()]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_equal_one_render(tmp_path):
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    out = str(tmp_path / "sum.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    sys.path.insert(0, os.path.join(ROOT, "embree-benchmark-protoray_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import scenes
    mesh, view = scenes.small_scene()
    O = oracle.Oracle()
    s = O.scene(mesh.positions, mesh.indices)
    W, H = 16, 12
    acc, rays = s.render(O.camera(view, W, H), W, H, 0, 4, 3, nthreads=1)
    np.testing.assert_allclose(got[:-1].reshape(acc.shape), acc, rtol=1e-12, atol=1e-12)
    assert got[-1] == rays
