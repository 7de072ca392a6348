"""GPU TD-MLWF through the C ABI against the oracle and the reference's jade_complex
test values: the six matrices, JADE, the rotation, centres and spreads."""
import json
import os

import numpy as np
import pytest
import torch

from helpers import rel_max, small_system
from wannier_cases import A, CENTRES, NR, check_value, gaussian_states, jade_case

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "jade_cases.json")


def _ham(pb, precision="fp64"):
    return pb.KSHamiltonian(np.eye(3) * A, NR, precision)


@pytest.mark.parametrize("idx", [0, 1])
def test_jade_golden_on_gpu(pb, oracle_mod, idx):
    case = json.load(open(GOLDEN))[idx]
    a, maxsweep, tol = jade_case(case)
    h = _ham(pb)
    ad = torch.as_tensor(a).cuda()
    u, adiag, sweeps = h.jade(ad, maxsweep, tol)
    u, adiag = u.cpu().numpy(), adiag.cpu().numpy()
    for chk in case["checks"]:
        assert check_value(chk, u, adiag) == pytest.approx(chk["value"], abs=5e-8), chk
    _, u_ref, ad_ref, sw_ref = oracle_mod.jade(a, maxsweep, tol)
    assert sweeps == sw_ref
    assert np.abs(u - u_ref).max() < 1e-12 and np.abs(adiag - ad_ref).max() < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mlwf_matrices_match_oracle(pb, oracle_mod, precision):
    o, psi, _ = gaussian_states(oracle_mod)
    h = _ham(pb, precision)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    a = h.mlwf_matrices(torch.as_tensor(psi).to(dt).cuda()).cpu().numpy()
    ref = o.mlwf_matrices(psi)
    assert np.abs(a - ref).max() < (1e-12 if precision == "fp64" else 2e-6)


def test_mlwf_matrices_random_states_32(pb, oracle_mod):
    """Delocalised states on the 32^3 cfg0 grid, M = 37 (partial output tiles)."""
    sysd = small_system(pb, n=32, M=37, seed=41, with_proj=False, ecut=10.0)
    o = oracle_mod.System(sysd["lattice"], sysd["nr"])
    h = pb.KSHamiltonian(sysd["lattice"], sysd["nr"], "fp64")
    a = h.mlwf_matrices(torch.as_tensor(sysd["psi"]).cuda()).cpu().numpy()
    assert np.abs(a - o.mlwf_matrices(sysd["psi"])).max() < 1e-12


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mlwf_step_matches_oracle(pb, oracle_mod, precision):
    o, psi, lat = gaussian_states(oracle_mod, seed=3)
    a = o.mlwf_matrices(psi)
    _, u, adiag, sw_ref = oracle_mod.jade(a)
    w_ref = o.mlwf_rotate(psi, u)
    c_ref = np.array([oracle_mod.mlwf_center(adiag, i, lat) for i in range(len(CENTRES))])
    s_ref = np.array([oracle_mod.mlwf_spread(adiag, i, lat) for i in range(len(CENTRES))])
    h = _ham(pb, precision)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = torch.as_tensor(psi).to(dt).cuda()
    centres, spreads, sweeps = h.mlwf_step_(x)
    if precision == "fp64":
        assert sweeps == sw_ref
        assert np.abs(centres - c_ref).max() < 1e-10 and np.abs(spreads - s_ref).max() < 1e-10
        assert rel_max(x.cpu().numpy(), w_ref) < 1e-10
    else:
        assert np.abs(centres - c_ref).max() < 1e-4 and np.abs(spreads - s_ref).max() < 1e-4


def test_mlwf_rotate_matches_numpy(pb):
    h = _ham(pb)
    rng = np.random.default_rng(9)
    M = 70
    psi = rng.standard_normal((h.N, M)) + 1j * rng.standard_normal((h.N, M))
    u = rng.standard_normal((M, M)) + 1j * rng.standard_normal((M, M))
    x = torch.as_tensor(psi).cuda()
    h.mlwf_rotate_(x, torch.as_tensor(u).cuda())
    assert rel_max(x.cpu().numpy(), psi @ u.conj().T) < 1e-13


def test_mlwf_output_file_format(pb, oracle_mod, tmp_path):
    """mlwf_properties::calculate's text (mlwf_properties.hpp:33-41)."""
    from pinq_b200.wannier import MLWFProperties

    _, psi, _ = gaussian_states(oracle_mod, seed=4)
    h = _ham(pb)
    props = MLWFProperties(h)
    with open(tmp_path / "mlwf_results.dat", "w") as f:
        centres, spreads = props.calculate(f, 6, torch.as_tensor(psi).cuda())
    lines = (tmp_path / "mlwf_results.dat").read_text().split("\n")
    assert lines[0] == "Time step: 7" and lines[1] == "MLWFs:"
    assert lines[2] == (f"  WF 1: {centres[0, 0]:g}     {centres[0, 1]:g}     {centres[0, 2]:g}     "
                        f"Spread: {spreads[0]:g}")


def test_jade_rejects_non_finite_matrices(pb):
    """A non-finite entry (an orbital block that blew up) ends JADE after its first sweep
    with INQB_ERR_NONFINITE instead of iterating on NaN."""
    h = pb.KSHamiltonian(np.eye(3) * 10.0, (16, 16, 16), "fp64")
    rng = np.random.default_rng(2)
    M = 6
    x = rng.standard_normal((6, M, M)) + 1j * rng.standard_normal((6, M, M))
    a = torch.as_tensor(x + np.conj(np.transpose(x, (0, 2, 1)))).to("cuda").contiguous()
    a[2, 1, 3] = float("nan")
    with pytest.raises(pb.InqbError) as e:
        h.jade(a, maxsweep=100)
    assert e.value.status == 5  # INQB_ERR_NONFINITE


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_sharded_mlwf_pieces_equal_whole_step(pb, oracle_mod, precision, tol):
    """The orbital-sharded TD-MLWF step's device pieces through the C ABI
    (inqb_mlwf_gram_block, inqb_orbital_norms, inqb_mlwf_finish, inqb_jade,
    inqb_rotate_block, inqb_mlwf_centres) with two ranks' blocks emulated in one
    process: every (row block, column block) of the Gram matrices as the circulation
    forms it, the rotation terms summed per owner.  Equals inqb_mlwf_step on all
    orbitals.  The exchange itself runs over gloo in tests/test_parallel_gloo.py."""
    o, psi, lat = gaussian_states(oracle_mod, seed=3)
    h = _ham(pb, precision)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = torch.as_tensor(psi).to(dt).cuda()
    whole = x.clone()
    c_ref, s_ref, sw_ref = h.mlwf_step_(whole)
    blocks = [x[:, :4].contiguous(), x[:, 4:].contiguous()]
    starts = [0, 4, 6]
    Z = torch.zeros((3, 6, 6), dtype=torch.complex128, device="cuda")
    for q in range(2):
        for r in range(2):
            Z[:, starts[q]:starts[q + 1], starts[r]:starts[r + 1]] = h.mlwf_gram_block(blocks[q], blocks[r])
    norms = torch.cat([h.orbital_norms(b) for b in blocks])
    a = h.mlwf_finish(Z, norms)
    u, adiag, sweeps = h.jade(a)
    R = u.conj().T.contiguous()
    out = []
    for s in range(2):
        acc = None
        for r in range(2):
            part = h.rotate_block(blocks[r], R[starts[r]:starts[r + 1], starts[s]:starts[s + 1]])
            acc = part if acc is None else acc + part
        out.append(acc)
    got = torch.cat(out, 1)
    centres, spreads = h.mlwf_centres(adiag)
    assert sweeps == sw_ref
    assert np.abs(centres - c_ref).max() < tol and np.abs(spreads - s_ref).max() < tol
    assert rel_max(got.cpu().numpy(), whole.cpu().numpy()) < (tol if precision == "fp64" else 1e-5)
