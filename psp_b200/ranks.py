"""One process per GPU: rank bookkeeping over torch.distributed.

Ranks never exchange data inside a solve; the only collectives are the
barrier and max-over-ranks timing reduction around a timed region and the
gather of batch solutions (``batch.solve_batch``).  The same helpers run on
NCCL (GPU ranks) and gloo (CPU ranks, used by the multi-rank tests).
"""
import datetime
import os


def from_env():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=300, local_rank=None):
    """Joins the process group of a torchrun launch (MASTER_ADDR/PORT set)."""
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local_rank)
        kw["device_id"] = torch.device("cuda", local_rank)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)


def _device():
    import torch.distributed as dist
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(x, ws):
    """The largest of every rank's x (a float); x itself when ws == 1."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
