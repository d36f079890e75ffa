"""Event-sharded 3D hybrid MLEM over several ranks (stripmlem.distributed.ShardedHybrid).

CPU: two gloo ranks drive ShardedHybrid over a stand-in whose
back-projection is the FP64 oracle's, each rank holding half of the frame
events of tests/golden/hybrid_small.npz; the image both ranks end with must
equal the oracle's single-process MLEM on all events.

GPU: two processes on one GPU, each running the library's kernels on its own
half of the responses, exchange their accumulators through host memory
(gloo); the result must match one process iterating over all responses.  The
kernels of the two processes never wait on each other: the exchange is on
the host.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from test_hybrid_oracle import golden_inputs, oracle_setup


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleHybridShard:
    """Stand-in with the split-iteration methods of HybridReconstruction,
    computed by the FP64 oracle on the CPU (test infrastructure only)."""

    def __init__(self, s, geo, w, sens, frames):
        self.s, self.geo, self.w, self.sens, self.frames = s, geo, w, sens, frames
        self.rho = np.ones((s.n_planes, s.n_rows, s.n_columns), np.float64)
        self.n_voxels = self.rho.size
        self.torch_device = "cpu"
        self.acc = None

    def set_accumulator(self, acc):
        self.acc = acc

    def accumulate(self):
        from oracle import hybrid as oh
        back, _ = oh.mlem(self.s, self.geo, self.w, self.sens, self.frames, 1, rho=self.rho,
                          f64=True)
        self.acc.copy_(torch.from_numpy(back.reshape(-1)).to(self.acc.dtype))

    def update(self):
        self.rho = self.acc.numpy().astype(np.float64).reshape(self.rho.shape)


def _prepared():
    from oracle import hybrid as oh
    z, cfg, m, resp, centers = golden_inputs()
    s = oracle_setup(cfg)
    res = oh.reconstruct(s, centers, m, resp, 0)
    return s, res


def _cpu_rank(rank, world, port, n_iter, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from stripmlem.distributed import ShardedHybrid
        s, res = _prepared()
        fr = res["frames"]
        half = len(fr) // world
        shard = OracleHybridShard(s, res["geo"], res["w"], res["sens"],
                                  fr[rank * half:(rank + 1) * half].copy())
        ShardedHybrid(shard, exchange="host")(n_iter)
        np.save(out.format(rank), shard.rho)
    finally:
        dist.destroy_process_group()


def test_sharded_hybrid_equals_single_process_oracle(tmp_path):
    from oracle import hybrid as oh
    out = str(tmp_path / "rho{}.npy")
    mp.start_processes(_cpu_rank, args=(2, free_port(), 2, out), nprocs=2, join=True,
                       start_method="spawn")
    s, res = _prepared()
    ref, _ = oh.mlem(s, res["geo"], res["w"], res["sens"], res["frames"], 2, f64=True)
    r0, r1 = np.load(out.format(0)), np.load(out.format(1))
    assert np.array_equal(r0, r1)  # the ranks hold the same image
    # the accumulator is binary32 (as the device's): agreement to its rounding
    assert np.linalg.norm(r0 - ref) / np.linalg.norm(ref) < 1e-6


def _gpu_rank(rank, world, port, n_iter, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from stripmlem import hybrid as hy
        from stripmlem.distributed import ShardedHybrid
        z, cfg, m, resp, centers = golden_inputs()
        n, n_planes, p, z_left, length, s_z, s_dl = cfg
        half = len(resp[0]) // world
        mine = tuple(a[rank * half:(rank + 1) * half] for a in resp)
        with hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as rec:
            rec.set_geometry_from_matrix(centers, m)
            rec.set_sensitivity()
            rec.set_responses(*mine)
            shd = ShardedHybrid(rec, exchange="host")
            shd(n_iter)
            np.save(out.format(rank), rec.rho)
            shd.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_sharded_hybrid_gpu_equals_single_process(tmp_path):
    from stripmlem import hybrid as hy
    out = str(tmp_path / "rho{}.npy")
    mp.start_processes(_gpu_rank, args=(2, free_port(), 3, out), nprocs=2, join=True,
                       start_method="spawn")
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    with hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as rec:
        rec.set_geometry_from_matrix(centers, m)
        rec.set_sensitivity()
        rec.set_responses(*resp)
        rec(3)
        single = rec.rho.astype(np.float64)
    r0, r1 = np.load(out.format(0)), np.load(out.format(1))
    assert np.array_equal(r0, r1)
    assert np.linalg.norm(r0 - single) / np.linalg.norm(single) < 1e-5
    ref = z["calc_rho"].astype(np.float64)
    assert np.linalg.norm(r0 - ref) / np.linalg.norm(ref) < 1e-4


@pytest.mark.gpu
def test_hybrid_split_step_equals_iterate():
    """hybrid_accumulate + hybrid_update is one hybrid_iterate step, with the
    context's own accumulator and with a caller's buffer."""
    from stripmlem import hybrid as hy
    z, cfg, m, resp, centers = golden_inputs()
    n, n_planes, p, z_left, length, s_z, s_dl = cfg
    with hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as a, \
            hy.HybridReconstruction(n, n, n_planes, p, z_left, length, s_z, s_dl) as b:
        for r in (a, b):
            r.set_geometry_from_matrix(centers, m)
            r.set_sensitivity()
            r.set_responses(*resp)
        a(2)
        b.accumulate()
        b.update()
        acc = torch.zeros(b.n_voxels, dtype=torch.float32, device="cuda:0")
        b.set_accumulator(acc)
        b.accumulate()
        assert float(acc.sum()) > 0
        b.update()
        b.set_accumulator(None)
        ra, rb = a.rho.astype(np.float64), b.rho.astype(np.float64)
        assert np.linalg.norm(ra - rb) / np.linalg.norm(ra) < 1e-6
