"""Orbital sharding over two processes on the CPU (gloo): every orbital lands on
exactly one rank, the all-reduced density equals the density of all orbitals,
and timings reduce by their maximum.  The density kernel is stood in for by
numpy here; the GPU path calls the library's inqb_density through the same
pinq_b200.parallel.sharded_density."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from pinq_b200.parallel import orbital_range


class _NumpyDensity:
    def density(self, psi, occ):
        rho = (np.abs(psi) ** 2 * np.asarray(occ)[None, :]).sum(1)
        return torch.tensor(rho, dtype=torch.float64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, M, out_dir):
    import datetime

    import torch.distributed as dist

    from pinq_b200.parallel import max_over_ranks, sharded_density

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(0)  # every rank builds the same full set
        psi = rng.standard_normal((500, M)) + 1j * rng.standard_normal((500, M))
        occ = rng.uniform(0.5, 2.0, M)
        first, count = orbital_range(M, world, rank)
        rho = sharded_density(_NumpyDensity(), psi[:, first:first + count], occ[first:first + count])
        t = max_over_ranks(1.0 + rank)
        np.save(os.path.join(out_dir, f"rho{rank}.npy"), rho.numpy())
        np.save(os.path.join(out_dir, f"t{rank}.npy"), np.array([t]))
    finally:
        dist.destroy_process_group()


def _reducer_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    from pinq_b200.parallel import density_reducer

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rho = torch.arange(6, dtype=torch.float64) * (rank + 1)
        out = density_reducer()(rho)
        assert out is rho  # in place, as the library's callback requires
        np.save(os.path.join(out_dir, f"red{rank}.npy"), rho.numpy())
    finally:
        dist.destroy_process_group()


def test_density_reducer_sums_in_place(tmp_path):
    """The exchange step of a sharded SCF step (KSHamiltonian.set_density_reducer)."""
    mp.start_processes(_reducer_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"red{r}.npy"), np.arange(6) * 3.0)


def test_orbital_range_partitions():
    for M in (0, 1, 7, 16, 128, 131):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                f, c = orbital_range(M, world, r)
                assert c >= 0
                seen.extend(range(f, f + c))
            assert seen == list(range(M))
    with pytest.raises(ValueError):
        orbital_range(4, 2, 2)


@pytest.mark.parametrize("M", [7, 16])
def test_sharded_density_two_ranks(tmp_path, M):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), M, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rng = np.random.default_rng(0)
    psi = rng.standard_normal((500, M)) + 1j * rng.standard_normal((500, M))
    occ = rng.uniform(0.5, 2.0, M)
    ref = (np.abs(psi) ** 2 * occ[None, :]).sum(1)
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"rho{r}.npy"), ref, rtol=1e-14, atol=0)
        assert float(np.load(tmp_path / f"t{r}.npy")[0]) == 2.0


class _TorchBlocks:
    """The three block operations of KSHamiltonian that sharded_orthonormalize_ calls,
    in torch FP64 on the CPU (the library's kernels do the same on the GPU)."""

    dV = 0.37

    def overlap_block(self, a, b):
        return self.dV * a.to(torch.complex128).conj().T @ b.to(torch.complex128)

    def cholesky_inverse_(self, S):
        U = torch.linalg.cholesky(S).conj().T  # S = U^H U, U upper
        S.copy_(torch.linalg.inv(U).triu())
        return S

    def rotate_block(self, a, R):
        return (a.to(torch.complex128) @ R).to(a.dtype)


def _ortho_main(rank, world, port, M, out_dir):
    import datetime

    import torch.distributed as dist

    from pinq_b200.parallel import sharded_orthonormalize_, sharded_overlap

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(3)  # every rank builds the same full set
        psi = torch.tensor(rng.standard_normal((300, M)) + 1j * rng.standard_normal((300, M)))
        first, count = orbital_range(M, world, rank)
        mine = psi[:, first:first + count].clone()
        S, counts = sharded_overlap(_TorchBlocks(), mine)
        sharded_orthonormalize_(_TorchBlocks(), mine)
        np.save(os.path.join(out_dir, f"S{rank}.npy"), S.numpy())
        np.save(os.path.join(out_dir, f"psi{rank}.npy"), mine.numpy())
        np.save(os.path.join(out_dir, f"counts{rank}.npy"), np.array(counts))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,M", [(2, 7), (2, 16), (3, 4)])
def test_sharded_orthonormalize_equals_whole_block(tmp_path, world, M):
    """The orbital-sharded orthonormalisation (block circulation for the overlap, an
    all-reduce of the M x M matrix, per-owner sums of the rotation terms) equals the
    orthonormalisation of all orbitals at once; (3, 4) leaves the last rank empty."""
    mp.start_processes(_ortho_main, args=(world, _free_port(), M, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rng = np.random.default_rng(3)
    psi = torch.tensor(rng.standard_normal((300, M)) + 1j * rng.standard_normal((300, M)))
    ops = _TorchBlocks()
    S_ref = ops.overlap_block(psi, psi)
    ref = ops.rotate_block(psi, ops.cholesky_inverse_(S_ref.clone())).numpy()
    parts = []
    for r in range(world):
        assert list(np.load(tmp_path / f"counts{r}.npy")) == [orbital_range(M, world, q)[1] for q in range(world)]
        assert np.allclose(np.load(tmp_path / f"S{r}.npy"), S_ref.numpy(), rtol=0, atol=1e-12 * ops.dV * 600)
        parts.append(np.load(tmp_path / f"psi{r}.npy"))
    got = np.concatenate(parts, axis=1)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    ovl = ops.dV * got.conj().T @ got
    assert np.abs(ovl - np.eye(M)).max() < 1e-12
