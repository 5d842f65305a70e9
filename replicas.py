"""Replica plumbing for bench.py --gpus N (one process per GPU, independent
copies of the job, no data exchange): the barrier around the timed region,
the maximum over ranks of a timing, and the whole-job rate.  Works on any
torch.distributed backend -- NCCL on GPUs, gloo on CPU (tests)."""

import torch
import torch.distributed as dist


def _device():
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier():
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x):
    """The largest value of x over all ranks (x itself on one process)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms_max):
    """Units processed by all ranks per second of the slowest rank."""
    return world * units_per_rank / (ms_max / 1000.0)
