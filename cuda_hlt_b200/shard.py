"""Running the chain on several GPUs of a node, one process per GPU.

Events are independent: the VELO path has no exchange step (the reference processes each
event of a batch on its own), so rank r takes its own contiguous range of events and no
collective touches the data. The only collectives are the barrier around the timed region
and the reduction of the elapsed time, taken as the maximum over the ranks (the slowest rank
ends the job). Per-rank work is fixed as ranks are added: weak scaling.
"""


def event_range(rank, events_per_rank):
    """(first event, number of events) of rank `rank`."""
    if rank < 0 or events_per_rank < 0:
        raise ValueError("rank and events_per_rank must be non-negative")
    return rank * events_per_rank, events_per_rank


def max_over_ranks(value, dist, device):
    """`value` reduced with MAX over the ranks of the default process group (float64)."""
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
