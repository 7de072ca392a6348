"""The orbital-sharded orthonormalisation's device pieces (inqb_overlap_block,
inqb_cholesky_inverse, inqb_rotate_block) through the C ABI.  Two ranks' blocks are
emulated in one process: every (row block, column block) of the overlap is formed
with inqb_overlap_block, as the block circulation of
pinq_b200.parallel.sharded_orthonormalize_ forms it across ranks, and each owner's
orbitals are the sum of the rotation terms of all blocks.  The result equals
inqb_orthonormalize of all orbitals at once.  The exchange itself (ring shift,
all-reduce, per-owner reduce) runs over gloo in tests/test_parallel_gloo.py."""
import numpy as np
import pytest
import torch

from helpers import rel_max, small_system

pytestmark = pytest.mark.gpu


def _blocks_orthonormalize(h, blocks):
    counts = [b.shape[1] for b in blocks]
    starts = np.concatenate([[0], np.cumsum(counts)]).astype(int)
    Mt = int(starts[-1])
    S = torch.zeros((Mt, Mt), dtype=torch.complex128, device="cuda")
    for q, bq in enumerate(blocks):
        for r, br in enumerate(blocks):
            S[starts[q]:starts[q + 1], starts[r]:starts[r + 1]] = h.overlap_block(bq, br)
    h.cholesky_inverse_(S)
    out = []
    for s in range(len(blocks)):
        acc = None
        for r, br in enumerate(blocks):
            part = h.rotate_block(br, S[starts[r]:starts[r + 1], starts[s]:starts[s + 1]])
            acc = part if acc is None else acc + part
        out.append(acc)
    return torch.cat(out, 1), S


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-6)])
def test_sharded_pieces_equal_whole_orthonormalize(pb, precision, tol):
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    s = small_system(pb, n=32, M=20, seed=21, with_proj=False)
    h = pb.KSHamiltonian(s["lattice"], s["nr"], precision)
    psi = torch.as_tensor(s["psi"]).to("cuda", dt)
    # blocks of 11 and 9 orbitals (INQ's partition of 20 over 2 ranks would be 10 + 10;
    # uneven blocks check the offsets), the second a strided view of a wider buffer
    wide = torch.zeros((h.N, 12), dtype=dt, device="cuda")
    wide[:, :9] = psi[:, 11:]
    blocks = [psi[:, :11].contiguous(), wide[:, :9]]
    got, U_inv = _blocks_orthonormalize(h, blocks)
    ref = h.orthonormalize_(psi.clone())
    torch.cuda.synchronize()
    got = got.cpu().numpy().astype(np.complex128)
    ref = ref.cpu().numpy().astype(np.complex128)
    assert rel_max(got, ref) <= tol, rel_max(got, ref)
    ovl = got.conj().T @ got * h.volume_element
    assert np.abs(ovl - np.eye(20)).max() <= 100 * tol
    assert np.abs(np.tril(U_inv.cpu().numpy(), -1)).max() == 0.0


def test_cholesky_inverse_rejects_a_dependent_set(pb):
    s = small_system(pb, n=32, M=4, seed=22, with_proj=False)
    h = pb.KSHamiltonian(s["lattice"], s["nr"], "fp64")
    psi = torch.as_tensor(s["psi"]).to("cuda")
    # a zero orbital: its row and column of the overlap are exactly zero, so the last
    # pivot is exactly 0 and zpotrf's test (pivot <= 0) rejects it.  A duplicated
    # orbital would leave a pivot of rounding size whose sign varies with the order of
    # the overlap's sums, accepted or rejected by chance, as by zpotrf itself.
    psi[:, 3] = 0
    S = h.overlap_block(psi, psi)
    with pytest.raises(RuntimeError, match="not positive definite"):
        h.cholesky_inverse_(S)


def test_rotate_block_rejects_overlapping_output(pb):
    s = small_system(pb, n=32, M=4, seed=23, with_proj=False)
    h = pb.KSHamiltonian(s["lattice"], s["nr"], "fp64")
    psi = torch.as_tensor(s["psi"]).to("cuda")
    R = torch.eye(4, dtype=torch.complex128, device="cuda")
    with pytest.raises(RuntimeError, match="overlaps"):
        h.rotate_block(psi, R, out=psi)
