"""Host-side helpers for running independent solves on several GPUs.

Solves are independent units: each rank (one process per GPU) takes its own
share of the work and no data-path collective is needed.  Timing is the
maximum over ranks."""


def assign(n_items, rank, world):
    """Round-robin share of ``n_items`` work units for ``rank`` of ``world``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank/world")
    return list(range(rank, n_items, world))


def max_over_ranks(value, dist=None, device="cpu"):
    """Maximum of a per-rank float over the process group (``value`` itself
    without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
