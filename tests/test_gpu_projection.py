"""The two forms of the KB projection of H|psi> (projector_all::project,
src/hamiltonian/projector_all.hpp:98-216) against the oracle, through the C ABI:

  * the projection fused into the first tile pass (the default) and the projection
    kernel of csrc/project.cu (mixed: tcgen05 TF32 tensor cores with the
    split-precision correction; FP64: CUDA cores) give H|psi> within the stated
    bounds of the FP64 oracle (FP64 1e-10 max-relative, mixed 1e-6 in norm);
  * orbital counts that fill no block (M = 70: a 64-orbital block and a ragged one;
    odd M: a half 16-byte piece), a strided block, a nonzero k + A (the coefficient
    table is rebuilt with the phases);
  * both forms are deterministic: two applies agree bit for bit;
  * an odd leading dimension (complex64 rows not 16-byte aligned) takes the fused form
    and is still right;
  * no device-side wait gave up (inqb_device_status).
"""
import numpy as np
import pytest
import torch

from helpers import make_oracle, make_product, rel_max, rel_norm, small_system

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-6}
DT = {"fp64": torch.complex128, "mixed": torch.complex64}


def _err(precision, out, ref):
    return rel_max(out, ref) if precision == "fp64" else rel_norm(out, ref)


@pytest.fixture(scope="module")
def sys70(pb):
    return small_system(pb, n=32, M=70, seed=31)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["kernel", "fused"])
def test_projection_modes_match_oracle(pb, oracle_mod, sys70, precision, mode):
    s = sys70
    o = oracle_mod.System(s["lattice"], s["nr"])
    kA = o.cart_to_cov(np.array([0.04, -0.03, 0.02]))
    o = make_oracle(oracle_mod, s, kA)
    h = make_product(pb, s, precision, kA)
    h.set_projection_mode(mode)
    x = torch.as_tensor(s["psi"]).to("cuda", DT[precision])
    out = h(x).cpu().numpy()
    h.device_status()
    err = _err(precision, out, o.apply_h(s["psi"]))
    assert err < TOL[precision], err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["kernel", "fused"])
def test_projection_is_deterministic(pb, sys70, precision, mode):
    h = make_product(pb, sys70, precision)
    h.set_projection_mode(mode)
    x = torch.as_tensor(sys70["psi"]).to("cuda", DT[precision])
    a = h(x)
    b = h(x)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["kernel", "fused"])
@pytest.mark.parametrize("M,lo,hi", [(7, 2, 9), (33, 0, 33), (4, 0, 3)])
def test_projection_ragged_and_strided(pb, oracle_mod, sys70, precision, mode, M, lo, hi):
    """Blocks [lo, hi) of a buffer of M + 3 orbitals: odd orbital counts (a half-filled
    16-byte piece), an offset block, and an odd leading dimension (7), whose complex64
    rows are not 16-byte aligned, so the mixed context takes the fused form."""
    s = sys70
    o = make_oracle(oracle_mod, s)
    h = make_product(pb, s, precision)
    h.set_projection_mode(mode)
    full = torch.as_tensor(s["psi"][:, :M + 3]).to("cuda", DT[precision])
    view = full[:, lo:hi]
    out = h(view).cpu().numpy()
    h.device_status()
    err = _err(precision, out, o.apply_h(s["psi"][:, lo:hi]))
    assert err < TOL[precision], err


def test_tensor_core_projection_close_to_fused(pb, sys70):
    """Mixed: the tensor-core projections and the fused FP32-product / FP64-sum ones
    give H|psi> within the FP32 rounding of each other."""
    h = make_product(pb, sys70, "mixed")
    x = torch.as_tensor(sys70["psi"]).to("cuda", torch.complex64)
    h.set_projection_mode("kernel")
    a = h(x).cpu().numpy()
    h.set_projection_mode("fused")
    b = h(x).cpu().numpy()
    assert rel_norm(a, b) < 5e-7


def test_output_takes_the_input_row_stride(pb, sys70):
    """The C ABI takes one leading dimension for input and output: a new output block
    gets the input's row stride, and an output with another stride is refused."""
    h = make_product(pb, sys70, "mixed")
    full = torch.as_tensor(sys70["psi"][:, :10]).to("cuda", torch.complex64)
    view = full[:, 2:9]
    out = h(view)
    assert out.shape == view.shape and out.stride(0) == view.stride(0)
    with pytest.raises(ValueError):
        h.apply(view, out=torch.empty_like(view.contiguous()))
