"""Sharding across ranks (one process per GPU).

Assembly: the (source, field, lag) blocks are independent, so each rank
assembles the rows of a contiguous range of source triangles for every field
triangle and lag (ebem_assemble_sa_panel); no data-path collective is needed.
Rank r of W takes sources [r N / W, (r + 1) N / W).  When one rank needs the
whole matrix, the panels are gathered into E[l][3 src0 : 3 (src0 + nsrc), :]
with one all-gather per lag.

Time marching on the panels (``march_panels``): E_0 is gathered once and
factorised on every rank; per step each rank forms its rows of the history
sum_{l>=1} E_l phi_{n-l} from its own panel (one HBM-bound GEMV over the
concatenated lags), one all-gather of those 3N values builds the
right-hand side, and every rank solves with E_0 (replicated, 3N unknowns) so
that phi_n is known everywhere for the next step.  Per step the exchange is
3N doubles; the E_l (the memory) stay split.
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


class DeviceOps:
    """The marching's compute steps on the device, through the C ABI."""

    def lu(self, A):
        from . import core
        return core.DeviceLU(A)

    def solve(self, lu, y):
        return lu.solve(y)

    def history(self, A, rows, x, y):
        from . import core
        return core.history_gemv(A, rows, x, y)


class HostOps:
    """The same steps with torch on the host (the gloo path of the tests)."""

    def lu(self, A):
        import torch
        return torch.linalg.lu_factor(A)

    def solve(self, lu, y):
        import torch
        y.copy_(torch.linalg.lu_solve(lu[0], lu[1], y.reshape(-1, 1)).reshape(-1))
        return y

    def history(self, A, rows, x, y):
        K = A.numel() // rows
        y -= A.reshape(K, rows).t() @ x
        return y


def march_panels(panel, rhs, n: int, world: int, rank: int, group=None, ops=None):
    """phi (nT, 3N), on every rank, from this rank's row panel of E_0..E_{L-1}
    (the buffer of ``core.assemble_sa_panel``: (L, 3N, 3 nsrc), column-major
    per lag) and the right-hand side rhs (nT, 3N).  ``ops`` selects device
    (default) or host compute."""
    import torch
    import torch.distributed as dist
    ops = ops or DeviceOps()
    L, n3, rows = panel.shape
    nT = rhs.shape[0]
    src0, nsrc = row_panel(rank, world, n)
    if rows != 3 * nsrc or n3 != 3 * n:
        raise ValueError("panel does not match this rank's rows")
    E0 = panel[0].t()                                   # [row, col] of this rank's rows
    if world > 1:
        E0 = gather_panels(E0.unsqueeze(0).contiguous(), n, world, group)[0]
    lu = ops.lu(E0.contiguous())
    sizes = [3 * row_panel(r, world, n)[1] for r in range(world)]
    width = max(sizes)
    rev = torch.zeros((nT, n3), dtype=torch.float64, device=panel.device)   # phi_n at row nT-1-n
    h = torch.zeros(width, dtype=torch.float64, device=panel.device)
    parts = [torch.empty_like(h) for _ in range(world)]
    for step in range(nT):
        h.zero_()
        M = min(step, L - 1)
        if M > 0:
            x = rev[nT - step:nT - step + M].reshape(-1)     # phi_{n-1}, ..., phi_{n-M}
            ops.history(panel[1:M + 1], rows, x, h[:rows])
        if world > 1:
            dist.all_gather(parts, h, group=group)
            hist = torch.cat([p[:sz] for p, sz in zip(parts, sizes)])
        else:
            hist = h[:rows]
        y = rhs[step] + hist
        ops.solve(lu, y)
        rev[nT - 1 - step] = y
    return torch.flip(rev, dims=[0])
