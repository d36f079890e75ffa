"""Event-sharded MLEM / OSEM over several ranks (stripmlem.distributed).

CPU: two gloo ranks drive ShardedReconstruction over a stand-in
reconstruction whose backprojection is the FP64 oracle's, each rank holding
half of the events; the image both ranks end with must equal the oracle's
single-process MLEM / OSEM on all events.  This covers the host side of the
multi-rank path: the split step, the all-reduce and the update order.

GPU: two processes on one GPU, each running the library's kernels on its own
half of the events, exchange their accumulators through host memory (gloo);
the result must match one process iterating over all events.  The kernels of
the two processes never wait on each other: the exchange is on the host.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import C1, C1_PHANTOM, PKG, ROOT
from oracle import oracle as orc

N_EVENTS = 6000   # divisible by 2 ranks x subsets, so e % M agrees on shards


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def c1_geometry():
    return orc.geometry(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"],
                        C1["p"], C1["s_z"], C1["s_dl"])


def c1_events(n, seed):
    import stripmlem as sm
    sc = sm.Scanner(C1["radius"], C1["length"], C1["n_y"], C1["n_z"], C1["p"], C1["p"],
                    C1["s_z"], C1["s_dl"])
    return sc, sm.generate_events(sc, C1_PHANTOM, n, seed=seed)


class OracleShard:
    """Stand-in with the split-iteration methods of stripmlem.Reconstruction,
    computed by the FP64 oracle on the CPU (test infrastructure only)."""

    def __init__(self, scanner, g, events):
        self.scanner = scanner
        self.g = g
        self.events = events
        self.torch_device = "cpu"
        self.rho = np.ones((g.n_y_pixels, g.n_z_pixels), np.float64)
        self.acc = None

    def set_accumulator(self, acc):
        self.acc = acc
        if acc is not None:
            acc.zero_()

    def accumulate(self, subset=0, n_subsets=1, mode=None):
        zu, zd, dl = (a[subset::n_subsets] for a in self.events)
        d = orc.forward_f64(self.g, zu, zd, dl, self.rho, self.g.sigma_z, self.g.sigma_dl)
        w = np.where(d > 0, 1.0 / np.where(d > 0, d, 1.0), 0.0)
        back = orc.adjoint_f64(self.g, zu, zd, dl, w, self.g.sigma_z, self.g.sigma_dl)
        self.acc += torch.from_numpy(back.reshape(-1))

    def update(self, scale=1.0):
        self.rho *= self.acc.numpy().reshape(self.rho.shape) * scale
        self.acc.zero_()


def _cpu_rank(rank, world, port, n_iter, n_subsets, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from stripmlem.distributed import ShardedReconstruction
        g = c1_geometry()
        sc, ev = c1_events(N_EVENTS, seed=21)
        half = N_EVENTS // world
        mine = tuple(a[rank * half:(rank + 1) * half] for a in ev)
        shard = OracleShard(sc, g, mine)
        ShardedReconstruction(shard, exchange="host")(n_iter, n_subsets)
        np.save(out.format(rank), shard.rho)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_subsets", [1, 2])
def test_sharded_iteration_equals_single_process_oracle(tmp_path, n_subsets):
    out = str(tmp_path / "rho{}.npy")
    mp.start_processes(_cpu_rank, args=(2, free_port(), 2, n_subsets, out), nprocs=2,
                       join=True, start_method="spawn")
    g = c1_geometry()
    _, (zu, zd, dl) = c1_events(N_EVENTS, seed=21)
    ref = orc.mlem_f64(g, zu, zd, dl, 2, n_subsets=n_subsets, sets_f32=True)
    r0, r1 = np.load(out.format(0)), np.load(out.format(1))
    assert np.array_equal(r0, r1)  # the ranks hold the same image
    assert np.linalg.norm(r0 - ref) / np.linalg.norm(ref) < 1e-12


def _gpu_rank(rank, world, port, n_iter, n_subsets, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import stripmlem as sm
        from stripmlem.distributed import ShardedReconstruction
        sc, ev = c1_events(N_EVENTS * 20, seed=22)
        half = len(ev[0]) // world
        mine = tuple(a[rank * half:(rank + 1) * half] for a in ev)
        with sm.Reconstruction(sc, device=0) as rec:
            rec.set_events(*mine)
            shd = ShardedReconstruction(rec, exchange="host")
            shd(n_iter, n_subsets)
            np.save(out.format(rank), rec.rho)
            shd.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("n_subsets", [1, 4])
def test_sharded_gpu_equals_single_process(tmp_path, n_subsets):
    import stripmlem as sm
    out = str(tmp_path / "rho{}.npy")
    mp.start_processes(_gpu_rank, args=(2, free_port(), 3, n_subsets, out), nprocs=2,
                       join=True, start_method="spawn")
    sc, ev = c1_events(N_EVENTS * 20, seed=22)
    with sm.Reconstruction(sc) as rec:
        rec.set_events(*ev, n_subsets=n_subsets)
        rec(None, 3)
        single = rec.rho.astype(np.float64)
    r0, r1 = np.load(out.format(0)), np.load(out.format(1))
    assert np.array_equal(r0, r1)
    # the shards' work items hold other events than one process's, so the
    # per-item fixed-point roundings differ: agreement at the accumulation's
    # own precision
    assert np.linalg.norm(r0 - single) / np.linalg.norm(single) < 5e-5
    g = c1_geometry()
    ref = orc.mlem_f64(g, *ev, 3, n_subsets=n_subsets, sets_f32=True)
    assert np.linalg.norm(r0 - ref) / np.linalg.norm(ref) < 1e-4


@pytest.mark.gpu
def test_split_step_equals_iterate():
    """strip_accumulate + strip_update on one context is one strip_iterate
    step, with the context's own accumulator and with a caller's buffer."""
    import stripmlem as sm
    sc, ev = c1_events(50_000, seed=23)
    with sm.Reconstruction(sc) as a, sm.Reconstruction(sc) as b:
        a.set_events(*ev)
        b.set_events(*ev)
        a(None, 2)
        b.accumulate()
        b.update(1.0)
        acc = torch.zeros(sc.total_n_pixels, dtype=torch.float64, device="cuda:0")
        b.set_accumulator(acc)
        b.accumulate()
        assert float(acc.sum()) > 0
        b.update(1.0)
        assert float(acc.abs().sum()) == 0.0  # the update consumes the accumulator
        b.set_accumulator(None)
        # the device-side binning places events in work items in an order
        # that varies from run to run, and with it the per-item roundings
        ra, rb = a.rho.astype(np.float64), b.rho.astype(np.float64)
        assert np.linalg.norm(ra - rb) / np.linalg.norm(ra) < 2e-5
