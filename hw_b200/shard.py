"""Placement of ZMWs on ranks (one process per GPU).

ZMWs, lanes and pools are independent through the whole chain (the reference
analyses each pool on its own, analyzer/BatchAnalyzer.cpp:149-375), so
several GPUs need no data exchange: each rank owns a disjoint ZMW range.
The only collectives are the timing barrier and the max-reduction of the
elapsed time.
"""


def lane_range(rank, world, total_lanes):
    """Contiguous share (first lane, lane count) of `total_lanes` for `rank`
    when a fixed set of lanes is divided among `world` ranks (strong
    scaling); the first total_lanes % world ranks take one lane more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(total_lanes, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def zmw_offset(rank, zmws_per_rank):
    """First global ZMW index of `rank` when every rank analyses a full chip
    of `zmws_per_rank` ZMWs (weak scaling)."""
    if rank < 0:
        raise ValueError("negative rank")
    return rank * zmws_per_rank


def max_over_ranks(x):
    """Maximum of a per-rank scalar over the process group (x itself when
    there is no group).  NCCL groups reduce on the current CUDA device."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
