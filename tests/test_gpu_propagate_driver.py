"""pinq_b200.propagate (real_time::propagate, src/real_time/propagate.hpp:33-140): the
time loop gives the same orbitals as the library steps called by hand, writes the
TD-MLWF lines and the results series, and resumes from its own checkpoint."""
import numpy as np
import pytest
import torch

from helpers import make_product, rel_max, small_system

pytestmark = pytest.mark.gpu


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def sysd(pb):
    return small_system(pb, n=32, M=4, seed=51, with_proj=False)


def _A(t):
    return (0.02 * np.sin(t), 0.0, 0.01)


def test_etrs_loop_matches_library_steps(pb, sysd):
    from pinq_b200 import propagate

    occ = np.full(4, 2.0)
    dt = 0.05
    h1 = make_product(pb, sysd, "fp64")
    x1 = _dev(sysd["psi"])
    res = propagate(h1, x1, occ, dt, 3, vector_potential=_A)
    h2 = make_product(pb, sysd, "fp64")
    x2 = _dev(sysd["psi"])
    for n in range(3):
        h2.etrs_step_(x2, dt, h2.cart_to_cov(_A(n * dt)), h2.cart_to_cov(_A((n + 1) * dt)))
    assert torch.equal(x1, x2)
    assert res.total_steps == 3 and res.time == [0.0, dt, 2 * dt, 3 * dt] and len(res.dipole) == 4
    eps = h2.band_energies(x2)
    assert res.total_energy[-1] == pytest.approx(float(np.dot(occ, eps)), rel=1e-12)


def test_lda_loop_matches_scf_steps(pb, sysd):
    from pinq_b200 import THEORY_LDA, propagate

    occ = np.full(4, 2.0)
    vion = _dev(sysd["V"], torch.float64)
    h1 = make_product(pb, sysd, "fp64")
    x1 = _dev(sysd["psi"])
    res = propagate(h1, x1, occ, 0.05, 2, vion=vion, theory=THEORY_LDA, vector_potential=_A)
    h2 = make_product(pb, sysd, "fp64")
    x2 = _dev(sysd["psi"])
    rho = h2.density(x2, occ)
    h2.ks_potential(rho, vion, THEORY_LDA, energies=False)
    for n in range(2):
        _, en = h2.etrs_scf_step_(x2, rho, 0.05, h2.cart_to_cov(_A(n * 0.05)), h2.cart_to_cov(_A((n + 1) * 0.05)),
                                  occ, vion, THEORY_LDA)
    assert rel_max(x1.cpu().numpy(), x2.cpu().numpy()) < 1e-13
    e_ref = float(np.dot(occ, h2.band_energies(x2))) - en["hartree"] - en["nvxc"] + en["xc"]
    assert res.total_energy[-1] == pytest.approx(e_ref, rel=1e-11)


def test_tdmlwf_lines_and_checkpoint_resume(pb, sysd, tmp_path):
    from pinq_b200 import propagate
    from pinq_b200.checkpoint import load_checkpoint

    occ = np.full(4, 2.0)
    dt = 0.05
    h1 = make_product(pb, sysd, "fp64")
    x1 = _dev(sysd["psi"])
    with open(tmp_path / "mlwf_results.dat", "w") as f:
        straight = propagate(h1, x1, occ, dt, 4, vector_potential=_A, tdmlwf=True, mlwf_out=f,
                             checkpoint_dir=str(tmp_path / "ck"), checkpoint_every=2)
    text = (tmp_path / "mlwf_results.dat").read_text()
    assert [ln for ln in text.split("\n") if ln.startswith("Time step")] == [f"Time step: {i}" for i in range(1, 5)]
    assert text.count("  WF ") == 16
    # the checkpoint of step 4 is the last one written; resume a copy from step 2
    h2 = make_product(pb, sysd, "fp64")
    x2 = _dev(sysd["psi"])
    with open(tmp_path / "m2.dat", "w") as f:
        propagate(h2, x2, occ, dt, 2, vector_potential=_A, tdmlwf=True, mlwf_out=f,
                  checkpoint_dir=str(tmp_path / "ck2"), checkpoint_every=2)
    h3 = make_product(pb, sysd, "fp64")
    x3 = torch.zeros_like(x2)
    res, occ3 = load_checkpoint(str(tmp_path / "ck2"), h3, x3)
    assert res.total_steps == 2 and np.array_equal(occ3, occ)
    with open(tmp_path / "m3.dat", "w") as f:
        resumed = propagate(h3, x3, occ3, dt, 4, vector_potential=_A, tdmlwf=True, mlwf_out=f, results=res,
                            start_step=2)
    # the TD-MLWF norms are FP64 atomic sums, so the resumed run agrees to rounding
    assert rel_max(x3.cpu().numpy(), x1.cpu().numpy()) < 1e-12
    assert resumed.time == straight.time and resumed.total_energy == pytest.approx(straight.total_energy, rel=1e-11)
