"""Orbital sharding across ranks (one process per GPU) and its one exchange.

H|psi> and the ETRS Taylor chains are independent per orbital once V and A are
shared, so a rank owns a contiguous block of orbitals and needs no data-path
collective for them.  The exchange is the density: each rank sums
occ |psi|^2 over its own orbitals and an all-reduce (SUM, FP64) completes it,
as INQ reduces the density over its states communicator
(src/observables/density.hpp:77-95 with the all-reduce of
src/parallel/communicator.hpp:116-188).  Collectives go through
torch.distributed: NCCL on GPUs, gloo on the CPU for tests.
"""
from __future__ import annotations


def orbital_range(M: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of rank's orbitals, INQ's block partition of the states
    (src/parallel/partition.hpp:33-95): blocks of ceil(M / world), the last ranks
    taking what is left (possibly nothing)."""
    if world < 1 or not (0 <= rank < world) or M < 0:
        raise ValueError("need world >= 1, 0 <= rank < world and M >= 0")
    bsize = (M + world - 1) // world
    first = min(bsize * rank, M)
    end = min(bsize * (rank + 1), M)
    return first, end - first


def allreduce_sum_(t, group=None):
    """In-place SUM over the ranks of group (no-op without an initialised group)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def max_over_ranks(x: float, device="cpu", group=None) -> float:
    """The largest value of x over the ranks (timings are reported this way)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sharded_density(ham, psi_local, occ_local, group=None):
    """Density of all ranks' orbitals: ham.density over this rank's block, then an
    FP64 all-reduce.  ham is anything with density(psi, occ) -> FP64 tensor [N]."""
    rho = ham.density(psi_local, occ_local)
    return allreduce_sum_(rho, group)


def density_reducer(group=None):
    """The exchange step of an orbital-sharded SCF step (KSHamiltonian.set_density_reducer):
    an in-place SUM of the density over the ranks, finished before it returns (the
    library's next kernels read the tensor on its own stream)."""
    import torch

    def reduce_(rho):
        allreduce_sum_(rho, group)
        if rho.is_cuda:
            torch.cuda.current_stream(rho.device).synchronize()
        return rho

    return reduce_
