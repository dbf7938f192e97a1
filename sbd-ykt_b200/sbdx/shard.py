"""Alpha-row shards of the product and of the Davidson solve over several
GPUs: one process per GPU, torch.distributed (NCCL) for the exchange.

The reference distributes W in 2-D blocks (an alpha block x a beta block per
rank), rotates the ket blocks between the ranks before each block product
(Mpi2dSlide, framework/mpi_utility.h:441-515; chemistry/tpb/mult.h:429-432,
599-607), sums the partial products (MpiAllreduce, mult.h:614-615) and
reduces every Davidson dot over the ranks (InnerProduct,
framework/dm_vector.h:179-243). The B200 form:

- rank r owns the contiguous alpha rows [a0_r, a1_r) of every vector (its
  part of W, HW and the subspace is (a1_r - a0_r) * nb elements, in the
  alpha-major order of the whole vector), the block boundaries multiples of 8
  and balanced by the work of the rows (`partition`);
- a product gathers the whole input into each GPU's HBM with one broadcast
  per rank (a variable-size all-gather over NVLink; the whole FP64 vector of
  the 400 M-determinant workload is 3.2 GB of 180 GB), then evaluates the
  rank's own rows completely (sbdx_sigma_rows_device), so no partial
  products are summed;
- the Davidson dots are local partial sums followed by one all-reduce, and
  the small Rayleigh-Ritz problem is solved on every rank from the same
  reduced numbers, so every rank takes the same steps.

`davidson` restates the FP64 reference form (chemistry/tpb/davidson.h:661-924
and the final energy of sbdiag.h:250-273) on these shards; `ShardedSigma` is
the product on one GPU of a multi-GPU job. The exchange goes through a `Comm`
(a torch.distributed group, or none at world size 1); the vector algebra of
the solver is torch arithmetic on the local rows.
"""
from __future__ import annotations

import time

import numpy as np


def partition(work, world: int, align: int = 8):
    """Contiguous blocks [a0, a1) of the rows 0 .. len(work)-1, one per rank,
    with about equal summed work; every a0 a multiple of `align` (the
    row-range product's alignment); blocks may be empty."""
    work = np.asarray(work, dtype=np.float64)
    n = len(work)
    cum = np.concatenate([[0.0], np.cumsum(work)])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        a = int(np.searchsorted(cum, target))
        a = min(n, max(bounds[-1], (a + align // 2) // align * align))
        bounds.append(a)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def row_work(ctx) -> np.ndarray:
    """Work of each alpha row of a context's product: its same-spin entries
    times nb, plus its alpha singles times all beta singles (the alpha-beta
    pairs), plus its beta same-spin entries (na x the beta list lengths,
    shared evenly over the rows)."""
    sa, da, _ = ctx.connectivity(0)
    sb, db, _ = ctx.connectivity(1)
    na, nb = len(sa), len(sb)
    beta_same = float((sb + db).sum())
    return (sa + da).astype(np.float64) * nb + sa.astype(np.float64) * float(sb.sum()) + beta_same


class Comm:
    """The exchange of a sharded solve over a torch.distributed group (NCCL
    for CUDA tensors, gloo for CPU ones); world size 1 without a group."""

    def __init__(self, group=None):
        self.dist = None
        self.rank, self.world = 0, 1
        if group is not None:
            import torch.distributed as dist

            self.dist = dist
            self.rank, self.world = dist.get_rank(), dist.get_world_size()

    def allreduce(self, t):
        """Sum of a tensor over the ranks, in place."""
        if self.dist is not None:
            self.dist.all_reduce(t)
        return t

    def gather_rows(self, full, local, bounds, nb: int):
        """Whole vector from the ranks' row blocks: `full` (na * nb) receives
        block r from rank r (a broadcast per rank; blocks differ in size)."""
        a0, a1 = bounds[self.rank]
        full[a0 * nb:a1 * nb].copy_(local)
        if self.dist is not None:
            for r, (b0, b1) in enumerate(bounds):
                if b1 > b0:
                    self.dist.broadcast(full[b0 * nb:b1 * nb], src=r)
        return full


class ShardedSigma:
    """Rank-local rows of S = H C on one GPU of a multi-GPU job: gathers the
    whole C into a device buffer, then evaluates rows [a0, a1) through the
    C-ABI (sbdx_sigma_rows_device)."""

    def __init__(self, ctx, comm: Comm, bounds, precision: int = 0):
        import torch

        import sbdx

        self.ctx, self.comm, self.bounds = ctx, comm, bounds
        self.precision = precision
        self.nb = ctx.nb
        dtype = torch.float64 if precision == sbdx.SBDX_FP64 else torch.float32
        self.full = torch.empty(ctx.na * ctx.nb, dtype=dtype, device="cuda")
        self.a0, self.a1 = bounds[comm.rank]

    def __call__(self, C_local, S_local):
        self.comm.gather_rows(self.full, C_local, self.bounds, self.nb)
        self.ctx.sigma_rows_device(self.precision, self.full.data_ptr(), S_local.data_ptr(), self.a0, self.a1)
        return S_local


def davidson(apply, hii_local, comm: Comm, W_local, max_it: int = 1, max_nb: int = 10, eps: float = 1e-4,
             max_time: float = 86400.0):
    """The FP64 reference Davidson (davidson.h:661-924) on row shards.

    apply(x_local, y_local) writes the rank's rows of H x; hii_local holds the
    rank's diagonal elements; W_local the rank's rows of the start vector
    (the whole vector has unit norm). Returns (energy, W_local, info) with
    info = {sigmas, residual, converged, seconds}; every rank returns the same
    energy, residual and step count. Dots: local sums, then one all-reduce
    per group of dots that the reference computes together."""
    import torch

    t0 = time.perf_counter()
    dev, n_loc = W_local.device, W_local.numel()
    C = torch.zeros((max_nb, n_loc), dtype=torch.float64, device=dev)
    HC = torch.zeros_like(C)
    H = np.zeros((max_nb, max_nb))
    W = W_local.clone()
    R = torch.empty_like(W)
    nsig, normR, done = 0, float("inf"), False
    steps = []

    def reduce(vals):
        t = torch.stack(vals) if isinstance(vals, (list, tuple)) else vals
        return comm.allreduce(t.clone()).cpu().numpy()

    for _ in range(max_it):
        if done:
            break
        C[0].copy_(W)
        for ib in range(max_nb):
            ts = time.perf_counter()
            apply(C[ib], HC[ib])
            nsig += 1
            hcol = reduce(C[:ib + 1] @ HC[ib])
            H[:ib + 1, ib] = hcol
            H[ib, :ib + 1] = hcol
            E, U = np.linalg.eigh(H[:ib + 1, :ib + 1])
            u = torch.tensor(U[:, 0], dtype=torch.float64, device=dev)
            E0 = float(E[0])
            W = u @ C[:ib + 1]
            R = E0 * W - u @ HC[:ib + 1]
            nw2, nr2 = reduce([W @ W, R @ R])
            normR = float(np.sqrt(nr2))
            W = W / np.sqrt(nw2)  # davidson.h:818-819
            if normR < eps:
                done = True
                break
            if ib < max_nb - 1:
                # preconditioned residual with the 1e-12 guard (davidson.h:855-862)
                den = E0 - hii_local
                v = (R / normR) / torch.where(den.abs() > 1e-12, den, den - 1e-12)
                for k in range(ib + 1):  # one pass of modified Gram-Schmidt
                    v -= float(reduce(C[k] @ v)) * C[k]
                v /= float(np.sqrt(reduce(v @ v)))
                C[ib + 1].copy_(v)
            steps.append(time.perf_counter() - ts)
            if time.perf_counter() - t0 + np.mean(steps) > max_time:  # davidson.h:876-903
                done = True
                break
    # final energy <W|HW> with one more product (sbdiag.h:250-273)
    HW = torch.empty_like(W)
    apply(W, HW)
    nsig += 1
    energy = float(reduce(W @ HW))
    info = {"sigmas": nsig, "residual": normR, "converged": bool(normR < eps),
            "seconds": time.perf_counter() - t0}
    return energy, W, info
