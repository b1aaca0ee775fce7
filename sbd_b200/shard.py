"""Alpha-row sharding of sigma and of the Davidson loop over several GPUs, one
process per GPU.

The reference distributes W and sigma in 2D blocks over an adet x bdet grid
of ranks (chemistry/tpb/helper.h:505-540, block ranges from get_mpi_range,
framework/mpi_utility.h:14-36).  Its mult moves ket blocks around a ring
(Mpi2dSlide, chemistry/tpb/mult.h:440-443, 612-621) and all-reduces sigma over
the task and row communicators (mult.h:630-631); its Davidson all-reduces
every inner product (framework/dm_vector.h:18-50).

Here rank k owns alpha rows [r0, r1) of every vector (the adet split; the
beta and task splits are not used).  A sigma gathers the full C on every rank
with one all-gather (NCCL over NVLink between GPUs, gloo on CPU), and each
rank then sums every term of its own rows on its own device
(sbdgpu_sigma_rows_device), so sigma needs no reduction.  Inner products are
one all-reduce of per-rank partial sums; the small projected eigenproblem is
solved redundantly on every rank from identical numbers.

The per-rank block sigma is a callable (full C, r0, r1) -> rows; on GPUs it
is ``gpu_block_sigma(ctx)``.
"""
from __future__ import annotations

import numpy as np


def mpi_range(size: int, rank: int, begin: int, end: int) -> tuple[int, int]:
    """The block of [begin, end) that rank `rank` of `size` owns: the first
    (end - begin) % size ranks take one element more (get_mpi_range,
    framework/mpi_utility.h:14-36)."""
    n = end - begin
    div, res = divmod(n, size)
    if rank < res:
        b = begin + (div + 1) * rank
        e = b + div + 1
    else:
        b = begin + (div + 1) * res + div * (rank - res)
        e = b + div
    return b, e


class AlphaRowShards:
    """Alpha-row blocks of na x nb vectors over the ranks of a process group."""

    def __init__(self, na: int, nb: int, group=None, adet_comm_size: int | None = None, bdet_comm_size: int = 1,
                 task_comm_size: int = 1):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        if bdet_comm_size != 1 or task_comm_size != 1:
            raise ValueError("the GPU path splits alpha rows only: bdet_comm_size and task_comm_size must be 1")
        if adet_comm_size not in (None, self.world):
            raise ValueError(f"adet_comm_size {adet_comm_size} must equal the number of ranks {self.world}")
        if na < self.world:
            raise ValueError(f"{na} alpha strings cannot be split over {self.world} ranks")
        self.na, self.nb = na, nb
        self.ranges = [mpi_range(self.world, k, 0, na) for k in range(self.world)]
        self.r0, self.r1 = self.ranges[self.rank]
        self.rows = self.r1 - self.r0
        self.max_rows = max(e - b for b, e in self.ranges)

    def local(self, full):
        """This rank's rows of a full vector."""
        return full[self.r0 * self.nb:self.r1 * self.nb]

    def gather(self, local):
        """The full vector from every rank's rows (one all-gather of equal,
        zero-padded blocks)."""
        import torch
        nb = self.nb
        pad = torch.zeros(self.max_rows * nb, dtype=local.dtype, device=local.device)
        pad[:self.rows * nb] = local
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        self.dist.all_gather(parts, pad, group=self.group)
        return torch.cat([p[:(e - b) * nb] for p, (b, e) in zip(parts, self.ranges)])

    def dot(self, x, y) -> float:
        import torch
        s = torch.dot(x.double(), y.double()).reshape(1)
        self.dist.all_reduce(s, group=self.group)
        return float(s.item())

    def sigma(self, local_C, block_sigma):
        """This rank's rows of H C."""
        return block_sigma(self.gather(local_C), self.r0, self.r1)


def gpu_block_sigma(ctx):
    """Per-rank block sigma on this rank's GPU (sbdgpu_sigma_rows_device): the
    full C (a CUDA tensor) in, this rank's rows out."""
    import torch

    def f(full, r0, r1):
        out = torch.empty((r1 - r0) * ctx.nb, dtype=torch.float64, device=full.device)
        ctx.sigma_rows_device(full.data_ptr(), out.data_ptr(), r0, r1)
        return out
    return f


def davidson(shards: AlphaRowShards, block_sigma, hii_local, W_local, max_it: int, max_nb: int, eps: float):
    """The reference's restarted Davidson for the lowest root
    (chemistry/tpb/davidson.h:661-923: block <= max_nb, collapse restart to the
    Ritz vector, diagonal preconditioner with eps_reg = 1e-12, modified
    Gram-Schmidt) on alpha-row shards, then E = <W|HW> from one more sigma
    (sbdiag.h:239-262).  Returns (E, this rank's rows of W, [(E0, tol) per
    step])."""
    import torch
    eps_reg = 1.0e-12
    W = W_local.double().clone()
    W /= np.sqrt(shards.dot(W, W))
    trace = []
    done = False
    for _ in range(max_it):
        C = [W.clone()]
        HC = []
        H = np.zeros((max_nb, max_nb))
        for ib in range(max_nb):
            HC.append(shards.sigma(C[ib], block_sigma))
            for jb in range(ib + 1):
                H[jb, ib] = H[ib, jb] = shards.dot(C[jb], HC[ib])
            E, U = np.linalg.eigh(H[:ib + 1, :ib + 1])
            u = U[:, 0]
            W = sum(float(u[k]) * C[k] for k in range(ib + 1))
            R = sum(float(u[k]) * HC[k] for k in range(ib + 1)) - float(E[0]) * W
            W /= np.sqrt(shards.dot(W, W))
            tol = np.sqrt(shards.dot(R, R))
            R /= tol
            trace.append((float(E[0]), float(tol)))
            if tol < eps:
                done = True
                break
            if ib < max_nb - 1:
                den = float(E[0]) - hii_local
                den = torch.where(den.abs() > eps_reg, den, den - eps_reg)
                x = R / den
                for kb in range(ib + 1):
                    x -= shards.dot(C[kb], x) * C[kb]
                x /= np.sqrt(shards.dot(x, x))
                C.append(x)
        if done:
            break
    e = shards.dot(W, shards.sigma(W, block_sigma))
    return e, W, trace
