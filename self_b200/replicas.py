"""Process-group plumbing for runs with one process per GPU.

The measured workloads do not exchange data between GPUs: a single solve fits
one B200, and ensemble instances are independent.  N GPUs therefore run N
replicas (or N disjoint shares of an ensemble) with no data-path collective;
the only collectives are a barrier around the timed region and a max over
ranks of the device-timed duration, as the reference's own diagnostics do with
MPI_ALLREDUCE (src/SELF_Mesh.f90:2230-2249).

Rank, world size and the rendezvous address come from the environment
(torchrun).  ``backend=None`` picks NCCL when CUDA is available, else gloo.
"""
import datetime
import os

import torch
import torch.distributed as dist


def env():
    """(rank, world, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend=None, timeout_s=120):
    """Join the process group when WORLD_SIZE > 1; returns (rank, world, local_rank)."""
    rank, world, local_rank = env()
    if world > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local_rank


def active():
    return dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1


def _device():
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier():
    if active():
        dist.barrier()


def max_over_ranks(x):
    """The largest value of x over all ranks (x on a single process)."""
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    if not active():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def deal(n_items, rank, world):
    """Round-robin share of n_items independent units (ensemble instances) for one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("deal: bad rank/world")
    return list(range(rank, n_items, world))


def aggregate_rate(units_per_rank, world, t_max_s):
    """Whole-job rate of a weak-scaled run: all ranks' units over the slowest rank's time."""
    if t_max_s <= 0:
        raise ValueError("aggregate_rate: non-positive time")
    return units_per_rank * world / t_max_s


def finalize():
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
