"""inqb_orthonormalize_noalloc against inqb_orthonormalize, both called through the
C ABI: the allocation-free variant takes its overlap, inverse-factor and status
scratch from a fixed device array instead of allocating it per call.  Two calls in
a row on different orbitals check that each call starts from cleared scratch.
This file is named to be collected last, after the tests that allocate."""
import ctypes

import numpy as np
import pytest
import torch

from helpers import rel_max, small_system

pytestmark = pytest.mark.gpu


def _ortho(pb, h, psi, name):
    from pinq_b200 import _lib

    psi = h._check(psi)
    _lib.call(name, h._h, ctypes.c_void_p(psi.data_ptr()), psi.shape[1], psi.stride(0),
              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return psi


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_noalloc_matches_allocating_entry_point(pb, precision, tol):
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    h = pb.KSHamiltonian(small_system(pb, n=32, M=1)["lattice"], (32, 32, 32), precision)
    for seed in (11, 12):  # two calls in a row reuse the same scratch
        s = small_system(pb, n=32, M=24, seed=seed, with_proj=False)
        psi = torch.as_tensor(s["psi"]).to("cuda", dt)
        ref = _ortho(pb, h, psi.clone(), "inqb_orthonormalize")
        out = _ortho(pb, h, psi.clone(), "inqb_orthonormalize_noalloc")
        torch.cuda.synchronize()
        ref = ref.cpu().numpy().astype(np.complex128)
        out = out.cpu().numpy().astype(np.complex128)
        assert rel_max(out, ref) <= tol, rel_max(out, ref)
        ovl = out.conj().T @ out * h.volume_element
        assert np.abs(ovl - np.eye(out.shape[1])).max() <= 100 * tol


def test_noalloc_rejects_too_many_orbitals(pb):
    from pinq_b200 import _lib

    h = pb.KSHamiltonian(small_system(pb, n=32, M=1)["lattice"], (32, 32, 32), "mixed")
    psi = torch.zeros((h.N, 257), dtype=torch.complex64, device="cuda")
    with pytest.raises(RuntimeError, match="at most 256 orbitals"):
        _ortho(pb, h, psi, "inqb_orthonormalize_noalloc")
    assert _lib.lib().inqb_last_error().decode().find("257") >= 0
