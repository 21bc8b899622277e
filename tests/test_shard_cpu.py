"""The N > 1 path on the CPU: two gloo ranks each assemble their source-row
panel (here with the oracle, the same blocks the device panel kernel
produces), gather the panels, and must reproduce the full assembly; the
panels partition the rows and the timing/count reductions of the benchmark
(sum of counts, max of times) behave as on NCCL."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_row_panels_partition():
    from elastodynamicebem_b200 import shard
    for n in (1, 7, 128, 1280):
        for w in (1, 2, 3, 8):
            spans = [shard.row_panel(r, w, n) for r in range(w)]
            assert spans[0][0] == 0 and sum(s for _, s in spans) == n
            assert all(a + b == c for (a, b), (c, _) in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        shard.row_panel(2, 2, 10)


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem, shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    m, prm = mesh.screen_uniform(3), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    N = m.numberTriangles
    L = O.num_blocks(m, prm)
    src0, nsrc = shard.row_panel(rank, world, N)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]          # (L, 3N, 3N) [l][row, col]
    panel = torch.tensor(full[:, 3 * src0:3 * (src0 + nsrc), :])     # this rank's rows
    E = shard.gather_panels(panel, N, world).numpy()
    cnt = torch.tensor([float(np.count_nonzero(np.abs(panel.numpy()).reshape(L, nsrc, 3, N, 3).sum(axis=(2, 4))))])
    dist.all_reduce(cnt)
    t = torch.tensor([float(rank + 1)])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        np.save(out, E)
        np.save(out + ".meta.npy", np.array([cnt.item(), t.item(),
                                             np.count_nonzero(np.abs(full).reshape(L, N, 3, N, 3).sum(axis=(2, 4)))]))
    dist.destroy_process_group()


def test_two_rank_gather_reproduces_full(tmp_path):
    import socket
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "E.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    E = np.load(out)
    cnt, tmax, cfull = np.load(out + ".meta.npy")
    m, prm = mesh.screen_uniform(3), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    full = O.assemble_sa(m, prm, 7, 0, O.num_blocks(m, prm), nthreads=1)[0]
    assert np.array_equal(E, full)
    assert cnt == cfull and tmax == 2.0


def _panel_raw(full, src0, nsrc):
    """This rank's rows of E_l[row, col] in the panel buffer layout
    (L, 3N, 3 nsrc): column-major per lag, leading dimension 3 nsrc."""
    import torch
    return torch.tensor(full[:, 3 * src0:3 * (src0 + nsrc), :]).transpose(1, 2).contiguous()


def _march_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem, shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    m, prm = mesh.screen_uniform(3), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    N = m.numberTriangles
    L = O.num_blocks(m, prm)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]
    b = torch.tensor(O.rhs(m, prm, 7, problem.DATUM_SCREEN_T4EXP).T.copy())       # (nT, 3N)
    src0, nsrc = shard.row_panel(rank, world, N)
    phi = shard.march_panels(_panel_raw(full, src0, nsrc), b, N, world, rank, ops=shard.HostOps())
    np.save(out + f".{rank}.npy", phi.numpy())
    dist.destroy_process_group()


def test_two_rank_panel_marching(tmp_path):
    """Marching on two ranks' row panels (one all-gather of the history per
    step) reproduces the oracle's serial marching on both ranks."""
    import socket
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "phi")
    mp.start_processes(_march_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    m, prm = mesh.screen_uniform(3), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 10)
    L = O.num_blocks(m, prm)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]
    ref = O.march(full, O.rhs(m, prm, 7, problem.DATUM_SCREEN_T4EXP)).T            # (nT, 3N)
    for r in range(2):
        phi = np.load(out + f".{r}.npy")
        assert np.linalg.norm(phi - ref) <= 1e-12 * np.linalg.norm(ref)


def test_single_rank_panel_marching():
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem, shard
    m, prm = mesh.screen_uniform(2), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 8)
    N = m.numberTriangles
    L = O.num_blocks(m, prm)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]
    b = O.rhs(m, prm, 7, problem.DATUM_SCREEN_T4EXP)
    phi = shard.march_panels(_panel_raw(full, 0, N), torch.tensor(b.T.copy()), N, 1, 0, ops=shard.HostOps())
    ref = O.march(full, b).T
    assert np.linalg.norm(phi.numpy() - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("case", ["graded", "prism"])
def test_balanced_row_panels(case):
    """Row panels balanced by non-null pair-lags (prefix sum of row_weights):
    the weights add up to the oracle's null-test census, the spans partition
    the rows, and every rank's work is within 5% of the mean on the graded
    screen and the prism, where equal row counts are not."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from elastodynamicebem_b200 import mesh, problem, shard
    if case == "graded":
        m, prm = mesh.screen_graded(16, 16), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 40)
    else:
        m, prm = mesh.prism_bar(1.0, 1.0, 3.0, 0.25), problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 40)
    L = O.num_blocks(m, prm)
    w = shard.row_weights(m, prm, L)
    assert int(w.sum()) == O.count_nonnull(m, prm, L)
    for world in (2, 4, 8):
        spans = [shard.row_panel(r, world, len(w), w) for r in range(world)]
        assert spans[0][0] == 0 and sum(s for _, s in spans) == len(w)
        assert all(a + b == c for (a, b), (c, _) in zip(spans, spans[1:]))
        work = np.array([w[a:a + b].sum() for a, b in spans], dtype=float)
        assert work.max() <= 1.05 * work.mean(), (world, work)


def _balanced_march_worker(rank, world, port, out, case):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    from elastodynamicebem_b200 import problem, shard
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    m, prm, datum = _balanced_case(case)
    N = m.numberTriangles
    L = O.num_blocks(m, prm)
    w = shard.row_weights(m, prm, L)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]
    b = torch.tensor(O.rhs(m, prm, 7, datum).T.copy())
    src0, nsrc = shard.row_panel(rank, world, N, w)
    panel = _panel_raw(full, src0, nsrc)
    E = shard.gather_panels(torch.tensor(full[:, 3 * src0:3 * (src0 + nsrc), :]), N, world, weights=w).numpy()
    phi = shard.march_panels(panel, b, N, world, rank, ops=shard.HostOps(), weights=w)
    np.save(out + f".{rank}.npy", phi.numpy())
    if rank == 0:
        np.save(out + ".E.npy", E)
    dist.destroy_process_group()


def _balanced_case(case):
    from elastodynamicebem_b200 import mesh, problem
    if case == "graded":
        return mesh.screen_graded(6, 4), problem.ProblemParams(1.0, 1.0, 2.0, 1.0, 12), problem.DATUM_SCREEN_T4EXP
    return mesh.prism_bar(1.0, 1.0, 3.0, 1.0), problem.ProblemParams(1.0, 1.0, 2.0, 2.0, 16), problem.DATUM_SCREEN_T4EXP


@pytest.mark.parametrize("case", ["graded", "prism"])
def test_two_rank_balanced_panels(tmp_path, case):
    """Two gloo ranks on work-balanced (unequal) row panels: the gathered
    panels equal the full assembly and the panel marching equals the oracle's
    serial marching within 1e-12 on both ranks."""
    import socket
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "phi")
    mp.start_processes(_balanced_march_worker, args=(2, port, out, case), nprocs=2, start_method="spawn", join=True)
    m, prm, datum = _balanced_case(case)
    L = O.num_blocks(m, prm)
    full = O.assemble_sa(m, prm, 7, 0, L, nthreads=1)[0]
    assert np.array_equal(np.load(out + ".E.npy"), full)
    ref = O.march(full, O.rhs(m, prm, 7, datum)).T
    for r in range(2):
        phi = np.load(out + f".{r}.npy")
        assert np.linalg.norm(phi - ref) <= 1e-12 * np.linalg.norm(ref)
