"""Independent replicas across ranks (one process per GPU).

The single-model oil-water step does not shard (its Krylov solve needs the
whole operator), so running on N GPUs means N replicas of the workload with
no data-path collective.  The only cross-rank step is the timing reduction:
the job's time is the slowest rank's, its work the sum over ranks.
"""

from __future__ import annotations


def reduce_timing(seconds: float, work: float, device=None):
    """Return (max seconds over ranks, summed work) with torch.distributed
    when it is initialised, else the local values."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(seconds), float(work)
    dev = device if device is not None else ("cuda" if dist.get_backend() == "nccl" else "cpu")
    t = torch.tensor([seconds], dtype=torch.float64, device=dev)
    w = torch.tensor([work], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w.item())
