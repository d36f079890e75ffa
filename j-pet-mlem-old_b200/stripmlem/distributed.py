"""Event-sharded MLEM / OSEM over several processes, one per GPU.

Events are independent within an iteration, so each rank holds its own shard
of the event list and the whole image.  One step per subset is

    backprojection of the rank's events into a binary64 accumulator
        (strip_accumulate)  ->  all-reduce(sum) of the accumulator over the
        ranks  ->  the same multiplicative update on every rank (strip_update)

so every rank ends each step with the image a single process would compute
from all events (up to the order of the binary64 sums).  The reference runs
this loop in one process and sums its per-thread images before the update
(src/2d/strip/reconstruction.h:109-154); the all-reduce is that sum across
processes.

``exchange="device"`` all-reduces the CUDA accumulator in place (NCCL over
NVLink); ``exchange="host"`` stages it through host memory, for process
groups whose backend works on CPU tensors (gloo).
"""
import torch
import torch.distributed as dist


class ShardedReconstruction:
    """Drives ``rec`` (a stripmlem.Reconstruction holding this rank's events,
    or an object with the same set_accumulator / accumulate / update
    methods) in lock-step with the other ranks of ``group``."""

    def __init__(self, rec, group=None, exchange="device"):
        if exchange not in ("device", "host"):
            raise ValueError("exchange must be 'device' or 'host'")
        self.rec = rec
        self.group = group
        self.exchange = exchange
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        n = rec.scanner.n_y_pixels * rec.scanner.n_z_pixels
        self.acc = torch.zeros(n, dtype=torch.float64, device=rec.torch_device)
        rec.set_accumulator(self.acc)

    def _sync(self):
        if self.acc.is_cuda:
            torch.cuda.current_stream(self.acc.device).synchronize()

    def _all_reduce(self):
        if self.world == 1:
            return
        if self.exchange == "device":
            dist.all_reduce(self.acc, op=dist.ReduceOp.SUM, group=self.group)
            self._sync()
        else:
            host = self.acc.cpu()
            dist.all_reduce(host, op=dist.ReduceOp.SUM, group=self.group)
            self.acc.copy_(host)
            self._sync()

    def step(self, subset=0, n_subsets=1, mode=None):
        """One subset update: accumulate, all-reduce, update (scale n_subsets)."""
        self.rec.accumulate(subset, n_subsets, mode)
        self._all_reduce()
        self.rec.update(float(n_subsets))

    def __call__(self, n_iterations=1, n_subsets=1, mode=None, progress=None,
                 n_iterations_so_far=0):
        """n_iterations MLEM (n_subsets == 1) or OSEM iterations; progress as
        Reconstruction.__call__ (called with (iteration, finished))."""
        for it in range(n_iterations):
            if progress is not None:
                progress(n_iterations_so_far + it, False)
            for s in range(n_subsets):
                self.step(s, n_subsets, mode)
            if progress is not None and progress(n_iterations_so_far + it, True) is True:
                break

    def close(self):
        self.rec.set_accumulator(None)


class ShardedHybrid:
    """The same lock-step for the 3D hybrid reconstruction: ``rec`` (a
    stripmlem.hybrid.HybridReconstruction holding this rank's responses, or
    an object with the same set_accumulator / accumulate / update methods and
    n_voxels / torch_device attributes) back-projects its events into a
    float32 accumulator, the ranks sum the accumulators, and every rank makes
    the sum its image (the reference's sum of per-thread images,
    src/3d/hybrid/reconstruction.h:369-376, across processes)."""

    def __init__(self, rec, group=None, exchange="device"):
        if exchange not in ("device", "host"):
            raise ValueError("exchange must be 'device' or 'host'")
        self.rec = rec
        self.group = group
        self.exchange = exchange
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.acc = torch.zeros(rec.n_voxels, dtype=torch.float32, device=rec.torch_device)
        rec.set_accumulator(self.acc)

    def _all_reduce(self):
        if self.world == 1:
            return
        if self.exchange == "device":
            dist.all_reduce(self.acc, op=dist.ReduceOp.SUM, group=self.group)
        else:
            host = self.acc.cpu()
            dist.all_reduce(host, op=dist.ReduceOp.SUM, group=self.group)
            self.acc.copy_(host)
        if self.acc.is_cuda:
            torch.cuda.current_stream(self.acc.device).synchronize()

    def __call__(self, n_iterations=1, progress=None):
        for it in range(n_iterations):
            if progress is not None:
                progress(it, False)
            self.rec.accumulate()
            self._all_reduce()
            self.rec.update()
            if progress is not None:
                progress(it, True)

    def close(self):
        self.rec.set_accumulator(None)
