"""GPU checkpoints through the C ABI: files byte-identical to the oracle's
restatement of INQ's layout (operations/io.hpp, systems/electrons.hpp), exact
round trips in both precisions, sharded states, and the error of a missing or short
file (io::load returns false)."""
import os

import numpy as np
import pytest
import torch

from helpers import make_product, small_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sysd(pb):
    return small_system(pb, n=32, M=6, seed=31, with_proj=False)


def _files(d):
    out = {}
    for root, _, names in os.walk(d):
        for n in names:
            p = os.path.join(root, n)
            out[os.path.relpath(p, d)] = open(p, "rb").read()
    return out


def test_fp64_files_match_layout_and_round_trip(pb, oracle_mod, sysd, tmp_path):
    h = make_product(pb, sysd, "fp64")
    psi = torch.as_tensor(sysd["psi"]).cuda()
    occ = np.array([2.0, 2.0, 2.0, 1.5, 0.5, 0.0])
    h.save_orbitals(str(tmp_path / "lib"), psi, occ)
    oracle_mod.save_orbitals_layout(str(tmp_path / "ref"), sysd["psi"], occ)
    a, b = _files(tmp_path / "lib"), _files(tmp_path / "ref")
    assert sorted(a) == sorted(b) and all(a[k] == b[k] for k in a)
    back = torch.zeros_like(psi)
    occ2 = h.load_orbitals(str(tmp_path / "ref"), back)
    assert torch.equal(back, psi) and np.array_equal(occ2, occ)


def test_mixed_widens_and_rounds_exactly(pb, oracle_mod, sysd, tmp_path):
    h = make_product(pb, sysd, "mixed")
    psi32 = torch.as_tensor(sysd["psi"]).to(torch.complex64).cuda()
    h.save_orbitals(str(tmp_path / "lib"), psi32)
    oracle_mod.save_orbitals_layout(str(tmp_path / "ref"), psi32.cpu().numpy().astype(np.complex128))
    a, b = _files(tmp_path / "lib"), _files(tmp_path / "ref")
    assert sorted(a) == sorted(b) and all(a[k] == b[k] for k in a)
    back = torch.zeros_like(psi32)
    assert h.load_orbitals(str(tmp_path / "lib"), back, with_occupations=False) is None
    assert torch.equal(back, psi32)


def test_sharded_blocks_and_strided_rows(pb, oracle_mod, sysd, tmp_path):
    """Two ranks' blocks (first_state 0 and 3) written into one directory read back as
    one set; the device block may be a column slice of a wider array (ld > M)."""
    h = make_product(pb, sysd, "fp64")
    wide = torch.zeros((h.N, 9), dtype=torch.complex128, device="cuda")
    wide[:, 1:7] = torch.as_tensor(sysd["psi"]).cuda()
    occ = np.arange(6, dtype=float)
    d = str(tmp_path / "ck")
    h.save_orbitals(d, wide[:, 1:4], occ[:3], first_state=0)
    h.save_orbitals(d, wide[:, 4:7], occ[3:], first_state=3)
    psi, occ2 = oracle_mod.load_orbitals_layout(d, h.N, 6)
    assert np.array_equal(psi, sysd["psi"]) and np.array_equal(occ2, occ)
    out = torch.zeros((h.N, 8), dtype=torch.complex128, device="cuda")
    h.load_orbitals(d, out[:, 2:5], first_state=3)
    assert torch.equal(out[:, 2:5].cpu(), torch.as_tensor(sysd["psi"][:, 3:6]))


def test_missing_and_short_files_fail(pb, sysd, tmp_path):
    h = make_product(pb, sysd, "fp64")
    psi = torch.as_tensor(sysd["psi"]).cuda()
    with pytest.raises(pb.InqbError) as e:
        h.load_orbitals(str(tmp_path / "nothing"), psi)
    assert e.value.status == 8
    d = str(tmp_path / "ck")
    h.save_orbitals(d, psi, np.ones(6))
    f = os.path.join(d, "kpin0000000000", "states", "0000000004_0000000000")
    data = open(f, "rb").read()
    open(f, "wb").write(data[: len(data) // 2])
    with pytest.raises(pb.InqbError) as e:
        h.load_orbitals(d, psi)
    assert e.value.status == 8


def test_density_round_trip(pb, sysd, tmp_path):
    h = make_product(pb, sysd, "mixed")
    rho = torch.rand(h.N, dtype=torch.float64, device="cuda")
    h.save_density(str(tmp_path), rho)
    raw = np.fromfile(str(tmp_path / "spin_density" / "0000000000"))
    assert np.array_equal(raw, rho.cpu().numpy())
    assert torch.equal(h.load_density(str(tmp_path)), rho)


def test_checkpoint_resume_continues_propagation(pb, sysd, tmp_path):
    """Two ETRS steps straight, and one step + checkpoint + load into a new context
    + one step, end in the same orbitals (resume)."""
    from pinq_b200.checkpoint import RealTimeResults, load_checkpoint, save_checkpoint

    occ = np.full(6, 2.0)
    k = np.zeros(3)
    h1 = make_product(pb, sysd, "fp64")
    a = torch.as_tensor(sysd["psi"]).cuda()
    b = a.clone()
    h1.etrs_step_(a, 0.05, k, k)
    h1.etrs_step_(a, 0.05, k, k)
    h1.etrs_step_(b, 0.05, k, k)
    res = RealTimeResults()
    res.record(0, 0.0, 0.0)
    res.record(1, 0.05, 0.0)
    save_checkpoint(str(tmp_path), h1, b, occ, h1.density(b, occ), res)
    h2 = make_product(pb, sysd, "fp64")
    c = torch.zeros_like(b)
    back, occ2 = load_checkpoint(str(tmp_path), h2, c)
    assert back.total_steps == 1 and np.array_equal(occ2, occ)
    h2.etrs_step_(c, 0.05, k, k)
    assert torch.equal(c, a)
