"""Multi-GPU runs of the tile executor: independent replicas, one process per GPU.

The tile schedule does not shard: every tile reads and writes the whole state, and a state
of up to 34 qubits (complex64, 128 GiB) fits one 180 GB GPU, so N GPUs run N independent
circuits.  The only cross-rank step is the timing reduction: each rank measures its own
device time, the job time is the maximum over ranks, and the whole-job throughput counts
the work of all ranks.
"""
from typing import List, Sequence


def max_over_ranks(values: Sequence[float], dist=None, device=None) -> List[float]:
    """Element-wise maximum of ``values`` over all ranks (identity without a process group).

    ``device`` is where the reduction tensor lives: a CUDA device for NCCL, None (CPU) for gloo.
    """
    vals = [float(v) for v in values]
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    import torch
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def whole_job_rate(units_per_rank: float, seconds: float, world: int) -> float:
    """Units per second over the whole job: every rank processed ``units_per_rank`` units and
    the slowest rank took ``seconds``."""
    if seconds <= 0:
        raise ValueError("job time must be positive")
    return units_per_rank * world / seconds
