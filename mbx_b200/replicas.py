"""Timing of replica runs: one process per GPU (torchrun), each rank
evaluating its own configurations (beads, boxes) with no data-path exchange.
A time is the maximum over ranks; a throughput is all ranks' units over that
time."""


def max_over_ranks(values, dist=None, device=None):
    """Element-wise maximum of a list of floats over the ranks of the default
    process group (the values themselves without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def throughput(units_per_rank, ms_max, world):
    """All ranks' units per second when every rank did units_per_rank in at
    most ms_max milliseconds (weak scaling)."""
    return world * units_per_rank / (ms_max * 1e-3)
