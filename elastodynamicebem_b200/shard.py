"""Sharding across ranks (one process per GPU).

Assembly: the (source, field, lag) blocks are independent, so each rank
assembles the rows of a contiguous range of source triangles for every field
triangle and lag (ebem_assemble_sa_panel); no data-path collective is needed.
The ranges are balanced by work: ``row_weights`` counts the non-null
pair-lags of every source row (the null test of
BEMenerg_coreSA_calcMatrixBlock.m:57-61, the unit of the assembly's cost) and
``balanced_spans`` cuts their prefix sum into W parts of nearly equal work
(equal row counts, [r N / W, (r + 1) N / W), when no weights are given).
When one rank needs the whole matrix, the panels are gathered into
E[l][3 src0 : 3 (src0 + nsrc), :] with one all-gather per lag.

Time marching on the panels (``march_panels``): E_0 is gathered once and
factorised on every rank; per step each rank forms its rows of the history
sum_{l>=1} E_l phi_{n-l} from its own panel (one HBM-bound GEMV over the
concatenated lags), one all-gather of those 3N values builds the
right-hand side, and every rank solves with E_0 (replicated, 3N unknowns) so
that phi_n is known everywhere for the next step.  Per step the exchange is
3N doubles; the E_l (the memory) stay split.
"""
from __future__ import annotations


def row_weights(mesh, prm, L: int, block: int = 256):
    """Non-null (field, lag) blocks of every source row over lags [0, L): the
    null test ((l - 1) c_S dt < d + maxL_i + maxL_j) and ((l + 1) c_P dt >=
    d - maxL_i - maxL_j) of BEMenerg_coreSA_calcMatrixBlock.m:57-61, d the
    centroid distance, evaluated as the device kernels evaluate it."""
    import numpy as np
    c, ml = np.asarray(mesh.center, np.float64), np.asarray(mesh.maxL, np.float64)
    n = len(c)
    lags = np.arange(L, dtype=np.float64)
    lo = (lags - 1) * prm.velS * prm.dt          # ((l - 1) c_S) dt
    hi = (lags + 1) * prm.velP * prm.dt          # ((l + 1) c_P) dt
    w = np.zeros(n, dtype=np.int64)
    for i0 in range(0, n, block):
        i = np.arange(i0, min(n, i0 + block))
        v = c[None, :, :] - c[i][:, None, :]     # field - source
        d = np.sqrt((v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1]) + v[..., 2] * v[..., 2])
        dmin = (d - ml[None, :]) - ml[i][:, None]
        dmax = (d + ml[None, :]) + ml[i][:, None]
        ok = (lo[None, None, :] < dmax[..., None]) & (hi[None, None, :] >= dmin[..., None])
        w[i] = ok.sum(axis=(1, 2))
    return w


def balanced_spans(weights, world: int) -> list:
    """[(src0, nsrc)] of `world` contiguous row ranges whose weight sums are
    as equal as row granularity allows: cut r sits where the prefix sum
    crosses r / world of the total (the nearer of the two rows around it);
    every range keeps at least one row."""
    import numpy as np
    w = np.asarray(weights, dtype=np.float64)
    n = len(w)
    if world < 1 or world > n:
        raise ValueError("need 1 <= world <= number of rows")
    cum = np.concatenate([[0.0], np.cumsum(w)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(cum, target))
        if k > 0 and abs(cum[k - 1] - target) <= abs(cum[min(k, n)] - target):
            k -= 1
        k = max(cuts[-1] + 1, min(k, n - (world - r)))
        cuts.append(k)
    cuts.append(n)
    return [(cuts[r], cuts[r + 1] - cuts[r]) for r in range(world)]


def row_panel(rank: int, world: int, n: int, weights=None) -> tuple[int, int]:
    """(src0, nsrc) of this rank's source rows: balanced by `weights`
    (row_weights) when given, else equal row counts."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    if weights is not None:
        if len(weights) != n:
            raise ValueError("one weight per source row")
        return balanced_spans(weights, world)[rank]
    src0 = rank * n // world
    return src0, (rank + 1) * n // world - src0


def _spans(n: int, world: int, weights=None) -> list:
    return balanced_spans(weights, world) if weights is not None else [row_panel(r, world, n) for r in range(world)]


def gather_panels(panel, n: int, world: int, group=None, weights=None):
    """All-gather the ranks' row panels (nlag, 3 nsrc_r, 3N) into the full
    (nlag, 3N, 3N) blocks on every rank (torch.distributed; NCCL for device
    tensors, gloo for host tensors).  `weights` as given to row_panel."""
    import torch
    import torch.distributed as dist
    nlag = panel.shape[0]
    sizes = [3 * s for _, s in _spans(n, world, weights)]
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


def march_panels(panel, rhs, n: int, world: int, rank: int, group=None, ops=None, weights=None):
    """phi (nT, 3N), on every rank, from this rank's row panel of E_0..E_{L-1}
    (the buffer of ``core.assemble_sa_panel``: (L, 3N, 3 nsrc), column-major
    per lag) and the right-hand side rhs (nT, 3N).  ``ops`` selects device
    (default) or host compute; ``weights`` the row split (row_panel)."""
    import torch
    import torch.distributed as dist
    ops = ops or DeviceOps()
    L, n3, rows = panel.shape
    nT = rhs.shape[0]
    src0, nsrc = row_panel(rank, world, n, weights)
    if rows != 3 * nsrc or n3 != 3 * n:
        raise ValueError("panel does not match this rank's rows")
    E0 = panel[0].t()                                   # [row, col] of this rank's rows
    if world > 1:
        E0 = gather_panels(E0.unsqueeze(0).contiguous(), n, world, group, weights)[0]
    lu = ops.lu(E0.contiguous())
    sizes = [3 * s for _, s in _spans(n, world, weights)]
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
