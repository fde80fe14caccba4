"""Replicas across GPUs: one process per GPU, each running its own independent FDTD job.

The stepping path does not shard (each simulation fits one B200), so the process group carries no field data: it only
brackets a timed region with barriers and takes the maximum of the ranks' timings, and the whole-job rate is the
units every rank processed divided by that maximum.  Ranks read RANK / WORLD_SIZE / LOCAL_RANK (and MASTER_ADDR /
MASTER_PORT for the rendezvous) from the environment, as torchrun sets them.  Backend 'nccl' on GPUs, 'gloo' on CPU.
"""
from __future__ import annotations

import datetime
import os

__all__ = ['ReplicaGroup', 'replica_env']


def replica_env():
    """(rank, world size, local rank) from the environment; (0, 1, 0) outside torchrun."""
    return (int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1)),
            int(os.environ.get('LOCAL_RANK', 0)))


class ReplicaGroup:
    """The process group of the replicas (none for a single process).  Every rank takes the same collective steps in
    the same order; the group's timeout ends a collective whose peers never arrive with an error instead of a hang."""

    def __init__(self, backend='nccl', timeout_s=300.0):
        self.rank, self.world, self.local = replica_env()
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist
            kwargs = {'timeout': datetime.timedelta(seconds=float(timeout_s))}
            if backend == 'nccl':
                kwargs['device_id'] = torch.device('cuda', self.local)
            dist.init_process_group(backend, **kwargs)
            self._dist = dist

    @property
    def is_root(self):
        return self.rank == 0

    def barrier(self):
        if self._dist is not None:
            self._dist.barrier()

    def reduce_max(self, value):
        """The maximum of a float over the ranks (float64 all-reduce)."""
        if self._dist is None:
            return float(value)
        import torch
        device = 'cuda' if self.backend == 'nccl' else 'cpu'
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job_rate(self, units_per_rank, seconds):
        """Units all ranks processed per second of the slowest rank (each rank processed units_per_rank)."""
        return self.world * float(units_per_rank) / float(seconds)

    def close(self):
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
