"""Batched uneven cells (cfg3: 16 cubic cells, grids from {24,32,40,48}^3, 8..64
orbitals, 2..16 atoms) in one CUDA graph: identical to applying H cell by cell, and
the FP64 result of sampled cells matches the oracle."""
import numpy as np
import pytest
import torch

from helpers import rel_max

pytestmark = pytest.mark.gpu


def _cells(pb, precision):
    from pinq_b200 import systems

    out = []
    for c in systems.cfg3_cells(seed=0):
        h = pb.KSHamiltonian(c["lattice"], c["nr"], precision)
        V = systems.gaussian_potential(c["lattice"], c["nr"], c["positions"])
        h.set_scalar_potential(V)
        h.set_gaussian_projectors(c["positions"])
        psi = systems.random_orbitals(c["lattice"], c["nr"], c["M"], 25.0, c["seed"])
        dt = torch.complex128 if precision == "fp64" else torch.complex64
        out.append(dict(h=h, V=V, psi=psi, x=torch.as_tensor(psi).to("cuda", dt), cell=c))
    return out


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_matches_cell_by_cell(pb, precision):
    cells = _cells(pb, precision)
    assert len({c["cell"]["nr"][0] for c in cells}) > 1  # uneven
    single = [c["h"](c["x"]) for c in cells]
    batch = pb.CellBatch([c["h"] for c in cells])
    outs = [torch.empty_like(c["x"]) for c in cells]
    for _ in range(3):  # capture once, replay twice
        batch.apply([c["x"] for c in cells], outs)
    torch.cuda.synchronize()
    tol = 1e-5 if precision == "mixed" else 1e-12  # atomics in the projector sums reorder roundings
    for a, b in zip(single, outs):
        assert rel_max(b.cpu().numpy(), a.cpu().numpy()) < tol


def test_batch_fp64_matches_oracle(pb, oracle_mod):
    cells = _cells(pb, "fp64")
    batch = pb.CellBatch([c["h"] for c in cells])
    outs = [torch.empty_like(c["x"]) for c in cells]
    batch.apply([c["x"] for c in cells], outs)
    torch.cuda.synchronize()
    for k in (0, 7, 15):
        c = cells[k]
        o = oracle_mod.System(c["cell"]["lattice"], c["cell"]["nr"])
        o.set_potential(c["V"])
        o.set_projectors(o.build_gaussian_kb(c["cell"]["positions"]))
        sub = np.ascontiguousarray(c["psi"][:, :4])
        ref = o.apply_h(sub)
        assert rel_max(outs[k].cpu().numpy()[:, :4], ref) < 1e-10


def test_every_schedule_gives_the_same_h(pb, oracle_mod):
    """H|psi> under every launch schedule the autotuner may pick (each ysplit with
    128 and 256 threads per pass) matches the oracle; the autotuner keeps one of them."""
    from helpers import make_oracle, make_product, rel_norm, small_system

    s = small_system(pb, n=32, M=8, seed=21)
    o = make_oracle(oracle_mod, s)
    ref = o.apply_h(s["psi"])
    h = make_product(pb, s, "mixed")
    x = torch.as_tensor(s["psi"]).to("cuda", torch.complex64)
    y1 = 4  # tiles per x-plane of the 32^3 grid (32 = 8 x 4)
    for ys in (1, 2, 4):
        for t in (128, 256):
            h.set_schedule(8, (ys, t, 256 if t == 128 else 128, t))
            out = h.apply(x).cpu().numpy().astype(np.complex128)
            assert rel_norm(out, ref) < 1e-6, (ys, t)
    sched = h.autotune(8)
    assert y1 % sched[0] == 0 and all(v in (128, 256) for v in sched[1:])
    out = h.apply(x).cpu().numpy().astype(np.complex128)
    assert rel_norm(out, ref) < 1e-6
    with pytest.raises(Exception):
        h.set_schedule(8, (3, 256, 256, 256))
    h.set_schedule(8, None)
