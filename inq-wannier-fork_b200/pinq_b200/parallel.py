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


def _peer(group, r):
    import torch.distributed as dist

    return r if group is None else dist.get_global_rank(group, r)


def _block_counts(M_local: int, device, group=None) -> list[int]:
    """Orbital counts of every rank's block (an all-gather of one integer)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return [int(M_local)]
    t = torch.tensor([int(M_local)], dtype=torch.int64, device=device)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [int(x.item()) for x in out]


def _ring_shift(blk, recv_count: int, group=None):
    """Send blk to the next rank and take a block of recv_count orbitals from the
    previous one (one step of the block circulation of
    src/parallel/block_array_iterator.hpp)."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    nxt, prv = _peer(group, (rank + 1) % world), _peer(group, (rank - 1) % world)
    recv = torch.empty((blk.shape[0], recv_count), dtype=blk.dtype, device=blk.device)
    ops = []
    if blk.shape[1] > 0:
        ops.append(dist.P2POp(dist.isend, torch.view_as_real(blk.contiguous()), nxt, group))
    if recv_count > 0:
        rr = torch.view_as_real(recv)
        ops.append(dist.P2POp(dist.irecv, rr, prv, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return recv


def sharded_overlap(ham, psi_local, group=None):
    """The full FP64 overlap dV Psi^H Psi of all ranks' orbitals, on every rank, as
    operations::overlap's set-parallel branch forms it (src/operations/overlap.hpp:47-72):
    the orbital blocks circulate around the ranks, each rank fills the rows of the
    block it holds against the columns of its own, and an all-reduce sums the
    zero-padded matrix.  Returns (S, counts)."""
    import torch
    import torch.distributed as dist

    counts = _block_counts(psi_local.shape[1], psi_local.device, group)
    starts = [sum(counts[:i]) for i in range(len(counts))]
    world = len(counts)
    rank = dist.get_rank(group) if world > 1 else 0
    Mt = sum(counts)
    S = torch.zeros((Mt, Mt), dtype=torch.complex128, device=psi_local.device)
    c0, c1 = starts[rank], starts[rank] + counts[rank]
    blk, src = psi_local, rank
    for step in range(world):
        if counts[src] > 0 and counts[rank] > 0:
            S[starts[src]:starts[src] + counts[src], c0:c1] = ham.overlap_block(blk, psi_local)
        if step < world - 1:
            src = (src - 1) % world
            blk = _ring_shift(blk, counts[src], group)
    allreduce_sum_(torch.view_as_real(S), group)
    return S, counts


def sharded_orthonormalize_(ham, psi_local, group=None):
    """operations::orthogonalize (src/operations/orthogonalize.hpp:25-32) of orbitals
    split over ranks in blocks: the overlap of all of them (sharded_overlap), its
    Cholesky factor S = U^H U and U^-1 on every rank (FP64, the same summed matrix
    everywhere), then Psi <- Psi U^-1 as operations::rotate's set-parallel branch does
    it (src/operations/rotate.hpp:100-125): each rank multiplies its block by its rows
    of U^-1 for every rank's columns, and those terms are summed on the owner.
    ham provides overlap_block, cholesky_inverse_ and rotate_block (KSHamiltonian does,
    through the C ABI).  psi_local is overwritten; it is returned."""
    import torch
    import torch.distributed as dist

    S, counts = sharded_overlap(ham, psi_local, group)
    ham.cholesky_inverse_(S)
    return _sharded_rotate_(ham, psi_local, S, counts, group)


def _sharded_rotate_(ham, psi_local, R, counts, group=None):
    """psi <- psi R for orbitals split in blocks (counts per rank), R [Mt, Mt] the same
    on every rank: each rank multiplies its block by its rows of R for every rank's
    columns, and those terms are summed on the owner (operations::rotate's
    set-parallel branch, src/operations/rotate.hpp:100-125)."""
    import torch
    import torch.distributed as dist

    world = len(counts)
    rank = dist.get_rank(group) if world > 1 else 0
    starts = [sum(counts[:i]) for i in range(world)]
    r0, r1 = starts[rank], starts[rank] + counts[rank]
    mine = None  # the sum for this rank's own orbitals; psi_local is read until the last term
    for s in range(world):
        if counts[s] == 0:
            continue
        cols = slice(starts[s], starts[s] + counts[s])
        if counts[rank] > 0:
            part = ham.rotate_block(psi_local, R[r0:r1, cols])
        else:
            part = torch.zeros((psi_local.shape[0], counts[s]), dtype=psi_local.dtype, device=psi_local.device)
        if world > 1:
            dist.reduce(torch.view_as_real(part), dst=_peer(group, s), op=dist.ReduceOp.SUM, group=group)
        if s == rank:
            mine = part
    if mine is not None:
        psi_local.copy_(mine)
    return psi_local


def sharded_mlwf_step_(ham, psi_local, group=None, maxsweep=100, tol=1e-8):
    """mlwf_properties::calculate (src/observables/mlwf_properties.hpp:28-44) for
    orbitals split over ranks in blocks.  The three weighted Gram matrices
    Z_d = Psi^H diag(e^{i 2 pi r_d / |a_d|}) Psi are formed block by block as the
    orbital blocks circulate around the ranks (as sharded_overlap does), then summed
    by an all-reduce; the norms are gathered the same way.  Every rank then forms the
    six matrices of tdmlwf_trans::update and runs JADE on the same summed input, so
    every rank holds the same rotation u, and Psi <- Psi u^H is summed on the owners.
    (The reference splits the basis instead and all-reduces the matrices over it,
    src/wannier/tdmlwf_trans.hpp:96-172.)  ham provides mlwf_gram_block, orbital_norms,
    mlwf_finish, jade, rotate_block and mlwf_centres (KSHamiltonian does, through the C
    ABI).  psi_local is rotated in place; returns (centres [Mt, 3], spreads [Mt], sweeps)."""
    import torch
    import torch.distributed as dist

    counts = _block_counts(psi_local.shape[1], psi_local.device, group)
    starts = [sum(counts[:i]) for i in range(len(counts))]
    world = len(counts)
    rank = dist.get_rank(group) if world > 1 else 0
    Mt = sum(counts)
    Z = torch.zeros((3, Mt, Mt), dtype=torch.complex128, device=psi_local.device)
    c0, c1 = starts[rank], starts[rank] + counts[rank]
    blk, src = psi_local, rank
    for step in range(world):
        if counts[src] > 0 and counts[rank] > 0:
            Z[:, starts[src]:starts[src] + counts[src], c0:c1] = ham.mlwf_gram_block(blk, psi_local)
        if step < world - 1:
            src = (src - 1) % world
            blk = _ring_shift(blk, counts[src], group)
    allreduce_sum_(torch.view_as_real(Z), group)
    norms = torch.zeros(Mt, dtype=torch.float64, device=psi_local.device)
    if counts[rank] > 0:
        norms[c0:c1] = ham.orbital_norms(psi_local)
    allreduce_sum_(norms, group)
    a = ham.mlwf_finish(Z, norms)
    u, adiag, sweeps = ham.jade(a, maxsweep, tol)
    _sharded_rotate_(ham, psi_local, u.conj().T.contiguous(), counts, group)
    centres, spreads = ham.mlwf_centres(adiag)
    return centres, spreads, sweeps
