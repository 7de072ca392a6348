"""The persistent batch launch (one kernel over work items taken from a device queue,
inqb_batch_set_mode PERSISTENT): equal to applying H cell by cell to rounding and
bitwise repeatable, for the cfg3 cells plus ragged orbital counts, cells without
projectors and a non-default first-pass split; the CUDA-graph form is bitwise equal;
the form autotuner picks one of the two and keeps correct outputs; a grid outside the
kernel falls back to the graph (AUTO) or is refused (PERSISTENT); and a wait that
cannot complete ends the launch after its time limit with INQB_ERR_TIMEOUT, after
which the batch works."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _make(pb, precision, lattice, nr, positions, M, seed, proj=True):
    from pinq_b200 import systems

    h = pb.KSHamiltonian(lattice, nr, precision)
    h.set_scalar_potential(systems.gaussian_potential(lattice, nr, positions))
    if proj:
        h.set_gaussian_projectors(positions)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = torch.as_tensor(systems.random_orbitals(lattice, nr, M, 25.0, seed)).to("cuda", dt)
    return h, x


def _cells(pb, precision):
    from pinq_b200 import systems

    cells = [_make(pb, precision, c["lattice"], c["nr"], c["positions"], c["M"], c["seed"])
             for c in systems.cfg3_cells(seed=0)]
    rng = np.random.default_rng(5)
    for n, M, proj in ((16, 5, False), (20, 13, True), (48, 33, True)):
        a = n * systems.SPACING
        pos = rng.uniform(0, a, (3, 3))
        cells.append(_make(pb, precision, systems.cubic(a), (n, n, n), pos, M, 900 + n, proj))
    return cells


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-6), ("fp64", 1e-14)])
def test_persistent_equals_cell_by_cell(pb, precision, tol):
    """The same tile bodies, compiled into the persistent kernel instead of their own
    kernels: equal to rounding (the compiler may contract a product into an FMA
    differently in the two), and bitwise repeatable from launch to launch."""
    cells = _cells(pb, precision)
    # one cell with the first pass on one CTA per x-plane instead of the default split
    cells[0][0].set_schedule(cells[0][1].shape[1], (1, 256, 256, 256))
    single = [h(x) for h, x in cells]
    batch = pb.CellBatch([h for h, _ in cells], mode="persistent")
    outs = [torch.empty_like(x) for _, x in cells]
    first = None
    for _ in range(3):
        for y in outs:
            y.fill_(float("nan"))
        batch.apply([x for _, x in cells], outs)
        batch.status()
        errs = [_rel(b, a) for a, b in zip(single, outs)]
        assert max(errs) < tol, errs
        if first is None:
            first = [y.clone() for y in outs]
        else:
            assert all(torch.equal(a, b) for a, b in zip(first, outs))
    info = batch.info()
    assert info["form"] == "persistent" and info["items"] > 0 and info["ctas"] > 0
    # the CUDA-graph form of the same batch
    batch.set_mode("graph")
    batch.apply([x for _, x in cells], outs)
    batch.status()
    assert batch.info()["form"] == "graph"
    for a, b in zip(single, outs):
        assert torch.equal(a, b)  # the graph replays the cells' own kernels


def test_form_autotune(pb):
    cells = _cells(pb, "mixed")[:6]
    single = [h(x) for h, x in cells]
    outs = [torch.empty_like(x) for _, x in cells]
    batch = pb.CellBatch([h for h, _ in cells])
    form, ms = batch.autotune_form([x for _, x in cells], outs)
    assert form in ("graph", "persistent") and ms["graph"] > 0 and ms["persistent"] > 0
    assert form == ("persistent" if ms["persistent"] < ms["graph"] else "graph")
    for y in outs:
        y.zero_()
    batch.apply([x for _, x in cells], outs)
    batch.status()
    assert batch.info()["form"] == form
    for a, b in zip(single, outs):
        assert _rel(b, a) < 1e-6


def test_grid_outside_the_kernel(pb):
    from pinq_b200 import systems

    a = 64 * systems.SPACING
    pos = np.array([[1.0, 2.0, 3.0], [5.0, 5.0, 5.0]])
    cells = [_make(pb, "mixed", systems.cubic(a), (64, 64, 64), pos, 8, 1),
             _make(pb, "mixed", systems.cubic(24 * systems.SPACING), (24, 24, 24), pos, 8, 2)]
    single = [h(x) for h, x in cells]
    outs = [torch.empty_like(x) for _, x in cells]
    batch = pb.CellBatch([h for h, _ in cells])  # AUTO
    batch.apply([x for _, x in cells], outs)
    batch.status()
    assert batch.info()["form"] == "graph"
    for s, o in zip(single, outs):
        assert torch.equal(s, o)
    strict = pb.CellBatch([h for h, _ in cells], mode="persistent")
    with pytest.raises(pb.InqbError) as e:
        strict.apply([x for _, x in cells], outs)
    assert e.value.status == 2  # INQB_ERR_UNSUPPORTED


def test_unreachable_wait_times_out(pb):
    from pinq_b200 import systems

    rng = np.random.default_rng(8)
    cells = []
    for n, M in ((24, 16), (32, 8)):
        a = n * systems.SPACING
        cells.append(_make(pb, "mixed", systems.cubic(a), (n, n, n), rng.uniform(0, a, (4, 3)), M, n))
    single = [h(x) for h, x in cells]
    outs = [torch.empty_like(x) for _, x in cells]
    batch = pb.CellBatch([h for h, _ in cells], mode="persistent")
    batch.set_wait_limit(0.05)
    batch.test_unreachable_wait(True)
    batch.apply([x for _, x in cells], outs)
    with pytest.raises(pb.InqbError) as e:
        batch.status()
    assert e.value.status == 7  # INQB_ERR_TIMEOUT
    # the device and the batch stay usable: the next plan runs every item
    batch.test_unreachable_wait(False)
    batch.apply([x for _, x in cells], outs)
    batch.status()
    for s, o in zip(single, outs):
        assert _rel(o, s) < 1e-6
