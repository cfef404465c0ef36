"""Row-block distribution (phg_b200/rowblocks.py) with two gloo ranks on the
CPU: the partition covers every row once, the halo exchange delivers the
owners' values, the distributed product equals the single-process product,
and the distributed Jacobi-PCG reaches the oracle's single-process solution
(iterations within 2, solution within 1e3 * rtol).  The ranks' dot products
sum in another order than one process's, so the last bits differ."""
import os
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT, load_golden


def _worker(rank, world, port, case, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from phg_b200 import rowblocks
    with np.load(os.path.join(ROOT, "tests", "golden", case + ".npz")) as z:
        G = {k: z[k] for k in z.files}
    ptr, cols, vals = G["rows_ptr"], G["rows_cols"], G["rows_vals"]
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        part = rowblocks.partition_by_nnz(ptr, world)
        r0, r1 = part[rank], part[rank + 1]
        lp = ptr[r0:r1 + 1] - ptr[r0]
        lc, lv = cols[ptr[r0]:ptr[r1]], vals[ptr[r0]:ptr[r1]]
        plan = rowblocks.HaloPlan(part, rank, lp, lc)
        n = len(ptr) - 1
        xg = np.cos(np.arange(n) * 0.37)
        xe = plan.exchange(torch.from_numpy(xg[r0:r1].copy())).numpy()
        halo_ok = np.array_equal(xe[plan.nloc:], xg[plan.halo])
        y = plan.matvec(lv, torch.from_numpy(xg[r0:r1].copy())).numpy()
        x, nits, res = rowblocks.pcg(plan, lv, G["diag"][r0:r1], G["rhs"][r0:r1], rtol=float(G["rtol"]))
        out[rank] = dict(part=part.tolist(), halo_ok=bool(halo_ok), nhalo=len(plan.halo), y=y, x=x.numpy(),
                         nits=nits, res=res)
    finally:
        dist.destroy_process_group()


def _run(case, world=2):
    port = 29500 + (os.getpid() * 7 + world) % 3000
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    return [out[r] for r in range(world)]


def test_partition_covers_rows():
    sys.path.insert(0, ROOT)
    from phg_b200.rowblocks import partition_by_nnz
    ptr = np.array([0, 5, 5, 9, 30, 31, 40, 41])
    for k in (1, 2, 3, 7):
        part = partition_by_nnz(ptr, k)
        assert part[0] == 0 and part[-1] == 7 and np.all(np.diff(part) >= 0) and len(part) == k + 1


def test_distributed_pcg_two_gloo_ranks(oracle):
    case = "p2_m5_kappa"
    G = load_golden(case)
    outs = _run(case)
    ptr, cols, vals = G["rows_ptr"], G["rows_cols"], G["rows_vals"]
    n = len(ptr) - 1
    assert all(o["halo_ok"] for o in outs) and all(o["nhalo"] > 0 for o in outs)
    xg = np.cos(np.arange(n) * 0.37)
    y = np.concatenate([o["y"] for o in outs])
    yo = oracle.spmv(ptr, cols, vals, xg)
    assert np.allclose(y, yo, rtol=1e-14, atol=1e-14 * np.abs(yo).max())
    x = np.concatenate([o["x"] for o in outs])
    assert outs[0]["nits"] == outs[1]["nits"]
    xo, no, _, _ = oracle.pcg(ptr, cols, vals, G["diag"], G["rhs"], rtol=float(G["rtol"]), btol=0.0, atol=0.0)
    assert abs(outs[0]["nits"] - no) <= 2
    assert np.linalg.norm(x - xo) <= 1e3 * float(G["rtol"]) * np.linalg.norm(xo)
