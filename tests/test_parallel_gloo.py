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


class _TorchMlwf(_TorchBlocks):
    """The TD-MLWF block operations of KSHamiltonian that sharded_mlwf_step_ calls, in
    torch FP64 on the CPU (the oracle's JADE and centre formulas)."""

    lattice = np.diag([5.0, 6.0, 7.0])
    nr = (6, 6, 6)

    def _weights(self):
        sym = [np.where(np.arange(n) >= (n + 1) // 2, np.arange(n) - n, np.arange(n)) / n for n in self.nr]
        f = np.stack(np.meshgrid(*sym, indexing="ij"), -1).reshape(-1, 3)
        L = self.lattice
        r = f @ L
        th = 2 * np.pi * r / np.linalg.norm(L, axis=1)[None, :]
        return torch.tensor(np.exp(1j * th))  # [N, 3]

    def mlwf_gram_block(self, a, b):
        w = self._weights()
        return torch.stack([a.conj().T @ (w[:, d:d + 1] * b) for d in range(3)])

    def orbital_norms(self, psi):
        return (psi.abs() ** 2).sum(0).to(torch.float64)

    def mlwf_finish(self, Z, norms):
        sc = 1.0 / torch.sqrt(norms[:, None] * norms[None, :])
        out = []
        for d in range(3):
            zh = Z[d].conj().T
            out += [0.5 * sc * (Z[d] + zh), sc * (Z[d] - zh) / 2j]
        return torch.stack(out)

    def jade(self, a, maxsweep, tol):
        import oracle

        _, u, adiag, sw = oracle.jade(a.numpy(), maxsweep, tol)
        return torch.tensor(u), torch.tensor(adiag), sw

    def mlwf_centres(self, adiag):
        import oracle

        ad = adiag.numpy()
        M = ad.shape[1]
        return (np.array([oracle.mlwf_center(ad, i, self.lattice) for i in range(M)]),
                np.array([oracle.mlwf_spread(ad, i, self.lattice) for i in range(M)]))


def _mlwf_states(M):
    rng = np.random.default_rng(5)
    ops = _TorchMlwf()
    N = int(np.prod(ops.nr))
    # Gaussians at random points, mixed by a random unitary (JADE un-mixes them)
    sym = [np.where(np.arange(n) >= (n + 1) // 2, np.arange(n) - n, np.arange(n)) / n for n in ops.nr]
    f = np.stack(np.meshgrid(*sym, indexing="ij"), -1).reshape(-1, 3)
    cols = []
    for _ in range(M):
        c = rng.uniform(-0.5, 0.5, 3)
        d = (f - c + 0.5) % 1.0 - 0.5
        r2 = ((d @ ops.lattice) ** 2).sum(1)
        cols.append(np.exp(-r2 / 2.0))
    psi = np.stack(cols, 1).astype(complex)
    q, _ = np.linalg.qr(rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M)))
    return torch.tensor(psi @ q), N


def _mlwf_main(rank, world, port, M, out_dir):
    import datetime

    import torch.distributed as dist

    from pinq_b200.parallel import sharded_mlwf_step_

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        psi, _ = _mlwf_states(M)
        first, count = orbital_range(M, world, rank)
        mine = psi[:, first:first + count].clone()
        c, sp, sw = sharded_mlwf_step_(_TorchMlwf(), mine, maxsweep=30)
        np.save(os.path.join(out_dir, f"c{rank}.npy"), c)
        np.save(os.path.join(out_dir, f"sp{rank}.npy"), sp)
        np.save(os.path.join(out_dir, f"psi{rank}.npy"), mine.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,M", [(2, 6), (3, 4)])
def test_sharded_mlwf_step_equals_whole_block(tmp_path, oracle_mod, world, M):
    """The orbital-sharded TD-MLWF step (Gram blocks circulated and all-reduced, the
    norms summed, JADE on every rank, the rotation summed on the owners) equals the step
    on all orbitals at once: centres, spreads and rotated orbitals."""
    from pinq_b200.parallel import sharded_mlwf_step_

    mp.start_processes(_mlwf_main, args=(world, _free_port(), M, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    psi, _ = _mlwf_states(M)
    whole = psi.clone()
    c_ref, sp_ref, _ = sharded_mlwf_step_(_TorchMlwf(), whole, maxsweep=30)
    parts = []
    for r in range(world):
        assert np.allclose(np.load(tmp_path / f"c{r}.npy"), c_ref, rtol=0, atol=1e-10)
        # (a spread of a few-point grid can be the square root of a small negative number)
        assert np.allclose(np.load(tmp_path / f"sp{r}.npy"), sp_ref, rtol=0, atol=1e-10, equal_nan=True)
        parts.append(np.load(tmp_path / f"psi{r}.npy"))
    got = np.concatenate(parts, 1)
    assert np.abs(got - whole.numpy()).max() <= 1e-10 * np.abs(whole.numpy()).max()
