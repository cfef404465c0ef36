"""Row-block distribution of an assembled system over several processes, one
per GPU: the host-side plan of the multi-GPU solve.

The reference distributes a matrix by contiguous blocks of rows: rank r owns
global rows partition[r] .. partition[r + 1] - 1 (MAP.partition,
include/phg/map.h:101).  A matrix-vector product first brings the entries of
x that a rank's rows reference but other ranks own (the "halo") into the
rank's own buffer -- one exchange per product (phgMatVec's scatter,
src/matvec.c:883,957) -- and every dot product ends with a sum over the
ranks (phgVecDot / phgVecNorm2, src/matvec.c:81,1227).

This module holds that plan:

  partition_by_nnz   row blocks of near-equal nonzero counts
  HaloPlan           the halo columns of a rank's rows, renumbered after its
                     own rows, and the send lists that mirror the other
                     ranks' requests (found with one all-to-all at set-up)
  HaloPlan.exchange  one all_to_all_single of the halo values per product
  pcg                the reference's Jacobi-PCG recurrence (solver_pcg,
                     src/solver-phg.c:485-604) on the distributed rows: one
                     halo exchange per product, the dot products of an
                     iteration summed over the ranks with one all-reduce of
                     two scalars (r.z and ||r||^2) and one of p.Ap

The exchange and sums go through torch.distributed (NCCL between GPUs, gloo
on CPU).  The local product here is a plain gather-and-segment-sum of the
rank's rows over its extended vector; on GPUs it is the library's SpMV on the
rank's rows with their columns renumbered to the extended vector.  The plan
is exercised by two gloo ranks on CPU (tests/test_rowblocks.py); every run on
the GPUs available here has one GPU, so the multi-GPU solve is unmeasured on
hardware.
"""
import numpy as np
import torch


def partition_by_nnz(ptr, nranks):
    """Row blocks (partition[0..nranks], partition[0] = 0, partition[-1] =
    n) whose nonzero counts differ by at most one row's."""
    ptr = np.asarray(ptr, np.int64)
    n = len(ptr) - 1
    targets = ptr[-1] * np.arange(1, nranks) / nranks
    cuts = np.searchsorted(ptr, targets, side="left")
    part = np.concatenate([[0], np.clip(cuts, 0, n), [n]]).astype(np.int64)
    return np.maximum.accumulate(part)


class HaloPlan:
    """Column renumbering and halo exchange of rank `rank`'s rows
    [part[rank], part[rank + 1]).  `cols` are the global columns of those
    rows (CSR with local row pointers `ptr`)."""

    def __init__(self, part, rank, ptr, cols, group=None):
        import torch.distributed as dist
        self.part = np.asarray(part, np.int64)
        self.rank = rank
        self.nranks = len(self.part) - 1
        r0, r1 = self.part[rank], self.part[rank + 1]
        self.nloc = int(r1 - r0)
        cols = np.asarray(cols, np.int64)
        own = (cols >= r0) & (cols < r1)
        halo = np.unique(cols[~own])                 # sorted: grouped by owner
        owner = np.searchsorted(self.part, halo, side="right") - 1
        self.recv_counts = np.bincount(owner, minlength=self.nranks).astype(np.int64)
        # local column ids: own rows first, then the halo in owner order
        self.local_cols = np.empty(len(cols), np.int64)
        self.local_cols[own] = cols[own] - r0
        self.local_cols[~own] = self.nloc + np.searchsorted(halo, cols[~own])
        self.ptr = np.asarray(ptr, np.int64)
        self.halo = halo
        # tell each owner which of its rows this rank needs
        counts = torch.from_numpy(self.recv_counts.copy())
        send_counts = torch.empty_like(counts)
        dist.all_to_all_single(send_counts, counts, group=group)
        self.send_counts = send_counts.numpy().astype(np.int64)
        req = torch.from_numpy(halo.copy())
        got = torch.empty(int(self.send_counts.sum()), dtype=torch.int64)
        dist.all_to_all_single(got, req, [int(c) for c in self.send_counts], [int(c) for c in self.recv_counts],
                               group=group)
        self.send_idx = got.numpy() - r0              # my rows the others need, by destination
        if len(self.send_idx) and (self.send_idx.min() < 0 or self.send_idx.max() >= self.nloc):
            raise ValueError("halo request outside the owner's rows")
        self.group = group
        self._rows = np.repeat(np.arange(self.nloc), np.diff(self.ptr))

    def exchange(self, x_loc):
        """[x_loc, the halo values] (float64 torch tensor of nloc + nhalo)."""
        import torch.distributed as dist
        send = x_loc[torch.from_numpy(self.send_idx)]
        recv = torch.empty(len(self.halo), dtype=x_loc.dtype)
        dist.all_to_all_single(recv, send, [int(c) for c in self.recv_counts],
                               [int(c) for c in self.send_counts], group=self.group)
        return torch.cat([x_loc, recv])

    def matvec(self, vals, x_loc):
        """y = A_rows x: one halo exchange, then the local rows' products."""
        xe = self.exchange(x_loc).numpy()
        prod = np.asarray(vals) * xe[self.local_cols]
        y = np.zeros(self.nloc)
        np.add.at(y, self._rows, prod)
        return torch.from_numpy(y)


def _allsum(vals, group):
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64)
    dist.all_reduce(t, group=group)
    return t.tolist()


def pcg(plan, vals, diag_loc, b_loc, x_loc=None, rtol=1e-10, btol=0.0, atol=0.0, maxit=10000):
    """Jacobi-PCG on the distributed rows (solver_pcg's recurrence and
    stopping rule).  Returns (x_loc, nits, residual)."""
    g = plan.group
    b = torch.as_tensor(np.asarray(b_loc, np.float64))
    D = torch.as_tensor(np.asarray(diag_loc, np.float64))
    x = torch.zeros_like(b) if x_loc is None else torch.as_tensor(np.array(x_loc, np.float64))
    bb, x1 = _allsum([float(b @ b), float(x.abs().sum())], g)
    rb = bb ** 0.5
    if rb < 10.0 * np.finfo(float).tiny:
        return torch.zeros_like(b), 0, 0.0
    n_global = float(plan.part[-1])
    r = b - plan.matvec(vals, x) if x1 / n_global >= 10.0 * np.finfo(float).tiny else b.clone()
    (rr,) = _allsum([float(r @ r)], g)
    r0 = residual = rr ** 0.5
    tol = max(r0 * rtol, rb * btol, atol)
    nits, rz1 = 0, 0.0
    p = torch.zeros_like(b)
    while residual > tol and nits < maxit:
        z = r / D
        nits += 1
        rz2 = rz1
        (rz1,) = _allsum([float(r @ z)], g)
        if nits == 1:
            p = z.clone()
        else:
            if rz2 == 0.0:
                break
            p = z + (rz1 / rz2) * p
        Ap = plan.matvec(vals, p)
        (pAp,) = _allsum([float(p @ Ap)], g)
        if pAp == 0.0:
            break
        alpha = rz1 / pAp
        x = x + alpha * p
        r = r - alpha * Ap
        (rr,) = _allsum([float(r @ r)], g)
        residual = rr ** 0.5
    return x, nits, residual
