"""Sharding of the assembly across ranks (one process per GPU).

The (source, field, lag) blocks are independent, so each rank assembles the
rows of a contiguous range of source triangles for every field triangle and
lag (ebem_assemble_sa_panel); no data-path collective is needed.  Rank r of
W takes sources [r N / W, (r + 1) N / W).  When one rank needs the whole
matrix (a single-GPU factorisation of E_0, for instance), the panels are
gathered into E[l][3 src0 : 3 (src0 + nsrc), :] with one all-gather per lag.
"""
from __future__ import annotations


def row_panel(rank: int, world: int, n: int) -> tuple[int, int]:
    """(src0, nsrc) of this rank's source rows."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    src0 = rank * n // world
    return src0, (rank + 1) * n // world - src0


def gather_panels(panel, n: int, world: int, group=None):
    """All-gather the ranks' row panels (nlag, 3 nsrc_r, 3N) into the full
    (nlag, 3N, 3N) blocks on every rank (torch.distributed; NCCL for device
    tensors, gloo for host tensors)."""
    import torch
    import torch.distributed as dist
    nlag = panel.shape[0]
    sizes = [3 * row_panel(r, world, n)[1] for r in range(world)]
    width = max(sizes)
    padded = torch.zeros((nlag, width, 3 * n), dtype=panel.dtype, device=panel.device)
    padded[:, :panel.shape[1]] = panel
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:, :s] for p, s in zip(parts, sizes)], dim=1)
