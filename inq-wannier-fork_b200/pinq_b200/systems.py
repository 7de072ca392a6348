"""Seeded synthetic systems with the shapes of the benchmark configurations.

No public dataset is involved: cells, atoms, potentials and orbitals are made
here from fixed seeds.  Pure numpy (input preparation, not the hot path).

  cfg0  cubic a=10.26, 8 atoms (diamond), 32^3, 32 orbitals, ecut 25 Ha
  cfg1  cubic a=20.52, 64 atoms (2x2x2 diamond), 64^3, 128 orbitals
  cfg2  cfg0 cell, 16 orbitals, ETRS dt=0.05, 200 steps, A_x ~ N(0, 0.01^2)
  cfg3  16 cubic cells, grids from {24,32,40,48}^3, 8..64 orbitals, 2..16 atoms
  cfg4  cubic a=30, 240 atoms on a jittered shell of radius 6.7, 144^3, ecut 30 Ha
"""
from __future__ import annotations

import numpy as np

DIAMOND_FRAC = np.array([
    [0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0],
    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75], [0.75, 0.75, 0.25],
])

SPACING = 0.320625  # 10.26 / 32


def diamond_positions(a_conv: float, reps: int = 1) -> np.ndarray:
    """Cartesian positions of a reps^3 supercell of the conventional diamond cell."""
    out = []
    for i in range(reps):
        for j in range(reps):
            for k in range(reps):
                out.append((DIAMOND_FRAC + np.array([i, j, k])) * a_conv)
    return np.concatenate(out, 0)


def sym(n: int) -> np.ndarray:
    i = np.arange(n)
    return np.where(i >= (n + 1) // 2, i - n, i)


def rvectors(lattice, nr) -> np.ndarray:
    """Cartesian position of every grid point, [N, 3], INQ's symmetric range."""
    lattice = np.asarray(lattice, float).reshape(3, 3)
    f = [sym(n) / n for n in nr]
    c = np.stack(np.meshgrid(*f, indexing="ij"), -1).reshape(-1, 3)
    return c @ lattice


def gaussian_potential(lattice, nr, positions, amplitude=-4.0, sigma=0.8) -> np.ndarray:
    """V(r) = sum_atoms sum_images amplitude * exp(-|r - R|^2 / (2 sigma^2))."""
    lattice = np.asarray(lattice, float).reshape(3, 3)
    r = rvectors(lattice, nr)
    V = np.zeros(len(r))
    pos = np.asarray(positions, float).reshape(-1, 3)
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            for k in (-1, 0, 1):
                shift = i * lattice[0] + j * lattice[1] + k * lattice[2]
                for p in pos:
                    d2 = ((r - (p + shift)) ** 2).sum(1)
                    m = d2 < (8 * sigma) ** 2
                    V[m] += amplitude * np.exp(-d2[m] / (2 * sigma * sigma))
    return V


def gaussian_potential_device(lattice, nr, positions, device="cuda", amplitude=-4.0, sigma=0.8):
    """gaussian_potential evaluated with torch on the device (FP64), for grids whose
    host evaluation would be slow; returns a numpy array [N]."""
    import torch

    lat = torch.tensor(np.asarray(lattice, float).reshape(3, 3), dtype=torch.float64, device=device)
    f = [torch.tensor(sym(n) / n, dtype=torch.float64, device=device) for n in nr]
    c = torch.stack(torch.meshgrid(*f, indexing="ij"), -1).reshape(-1, 3)
    r = c @ lat
    V = torch.zeros(r.shape[0], dtype=torch.float64, device=device)
    pos = torch.tensor(np.asarray(positions, float).reshape(-1, 3), dtype=torch.float64, device=device)
    cut2 = (8 * sigma) ** 2
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            for k in (-1, 0, 1):
                shift = i * lat[0] + j * lat[1] + k * lat[2]
                for p in pos:
                    d2 = ((r - (p + shift)) ** 2).sum(1)
                    V += torch.where(d2 < cut2, amplitude * torch.exp(-d2 / (2 * sigma * sigma)),
                                     torch.zeros_like(d2))
    return V.cpu().numpy()


def random_orbitals_device(ham, M, ecut=25.0, seed=0):
    """random_orbitals built on the device with the library: complex N(0,1)
    plane-wave coefficients for 1/2|G|^2 <= ecut, the library's inverse FFT, then
    its FP64 orthonormalisation.  A torch tensor [N, M] in the context precision."""
    import torch

    nx, ny, nz = ham.nr
    recip = 2 * np.pi * np.linalg.inv(np.asarray(ham.lattice, float).reshape(3, 3)).T
    n = np.stack(np.meshgrid(sym(nx), sym(ny), sym(nz), indexing="ij"), -1).reshape(-1, 3)
    mask = 0.5 * ((n @ recip) ** 2).sum(1) <= ecut
    g = torch.Generator(device=ham.device).manual_seed(int(seed))
    coef = torch.randn((ham.N, M, 2), generator=g, device=ham.device, dtype=torch.float32)
    box = torch.view_as_complex(coef).to(ham.dtype) / np.sqrt(2.0)
    box *= torch.as_tensor(mask, device=ham.device)[:, None]
    psi = ham.to_real(box)
    del box, coef
    return ham.orthonormalize_(psi)


def orthonormalize(psi: np.ndarray, dV: float) -> np.ndarray:
    """psi U^-1 with dV psi^H psi = U^H U."""
    import scipy.linalg as sla
    S = dV * (psi.conj().T @ psi)
    U = sla.cholesky(S, lower=False)
    return sla.solve_triangular(U, psi.T, trans="T", lower=False).T


def random_orbitals(lattice, nr, M, ecut=25.0, seed=0, dtype=np.complex128) -> np.ndarray:
    """M orbitals with complex N(0,1) plane-wave coefficients for 1/2|G|^2 <= ecut,
    transformed to real space and orthonormalised with dV.  [N, M]."""
    lattice = np.asarray(lattice, float).reshape(3, 3)
    recip = 2 * np.pi * np.linalg.inv(lattice).T
    nx, ny, nz = nr
    n = np.stack(np.meshgrid(sym(nx), sym(ny), sym(nz), indexing="ij"), -1).reshape(-1, 3)
    G = n @ recip
    mask = 0.5 * (G ** 2).sum(1) <= ecut
    rng = np.random.default_rng(seed)
    ng = int(mask.sum())
    coef = (rng.standard_normal((ng, M)) + 1j * rng.standard_normal((ng, M))) / np.sqrt(2.0)
    box = np.zeros((nx * ny * nz, M), np.complex128)
    box[mask] = coef
    psi = np.fft.ifftn(box.reshape(nx, ny, nz, M), axes=(0, 1, 2)).reshape(-1, M)
    dV = abs(np.linalg.det(lattice)) / (nx * ny * nz)
    psi = orthonormalize(psi, dV)
    return np.ascontiguousarray(psi.astype(dtype))


def cubic(a: float) -> np.ndarray:
    return np.eye(3) * a


def shell_positions(n_atoms: int = 240, radius: float = 6.7, jitter: float = 0.05, center=(15.0, 15.0, 15.0),
                    seed: int = 0) -> np.ndarray:
    """Atoms on a jittered closed shell (the 240-atom fullerene-like cage of the
    large-cell configuration): n points of a golden-angle (Fibonacci) spiral on the
    sphere, each moved by N(0, jitter^2) per coordinate.  The spiral stands in for a
    fullerene's exact geometry, which the configuration does not give."""
    rng = np.random.default_rng(seed)
    k = np.arange(n_atoms) + 0.5
    z = 1.0 - 2.0 * k / n_atoms
    r = np.sqrt(1.0 - z * z)
    phi = k * np.pi * (3.0 - np.sqrt(5.0))
    unit = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    return np.asarray(center, float)[None, :] + radius * unit + rng.normal(0.0, jitter, (n_atoms, 3))


def config(name: str, M: int | None = None, seed: int = 0) -> dict:
    """Synthetic inputs of a named configuration (positions, V, orbitals, ...)."""
    if name in ("cfg0", "cfg2"):
        a, reps, n = 10.26, 1, 32
        M = M or (32 if name == "cfg0" else 16)
    elif name == "cfg1":
        a, reps, n = 20.52, 2, 64
        M = M or 128
    else:
        raise ValueError(name)
    lattice = cubic(a)
    nr = (n, n, n)
    pos = diamond_positions(10.26, reps)
    V = gaussian_potential(lattice, nr, pos)
    psi = random_orbitals(lattice, nr, M, 25.0, seed)
    out = dict(name=name, lattice=lattice, nr=nr, positions=pos, V=V, psi=psi, M=M,
               radius=3.0, sigma=1.0, ekb_s=1.5, ekb_p=-0.7)
    if name == "cfg2":
        rng = np.random.default_rng(seed + 1)
        out.update(dt=0.05, steps=200, amplitudes=rng.normal(0.0, 0.01, 200), occ=np.full(M, 2.0),
                   checkpoint_every=20)
    return out


def cfg3_cells(seed: int = 0, ncells: int = 16):
    """16 uneven cubic cells: grid n in {24,32,40,48}, edge n*SPACING, 8..64 orbitals
    (multiples of 8), 2..16 atoms placed uniformly at random with >= 2 bohr separation."""
    rng = np.random.default_rng(seed)
    cells = []
    for c in range(ncells):
        n = int(rng.choice([24, 32, 40, 48]))
        a = n * SPACING
        M = int(rng.integers(1, 9)) * 8
        na = int(rng.integers(2, 17))
        pos = []
        while len(pos) < na:
            p = rng.uniform(0, a, 3)
            ok = True
            for q in pos:
                d = p - q
                d -= a * np.round(d / a)
                if np.linalg.norm(d) < 2.0:
                    ok = False
                    break
            if ok:
                pos.append(p)
        cells.append(dict(lattice=cubic(a), nr=(n, n, n), positions=np.array(pos), M=M, seed=seed * 100 + c))
    return cells
