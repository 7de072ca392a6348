"""Non-finite inputs are rejected with INQB_ERR_NONFINITE (status 5) before any device
work or state change: the local potential, the vector potential and the kick field.
A non-finite time step is rejected as an invalid argument (status 1).  The reference
aborts on bad input (asserts, gpu::check_error); the library returns the status, and
the context keeps its previous state and stays usable."""
import numpy as np
import pytest
import torch

from helpers import make_product, small_system

pytestmark = pytest.mark.gpu


def test_nonfinite_inputs_are_rejected_and_the_context_stays_usable(pb):
    sysd = small_system(pb, n=32, M=2, seed=3, with_proj=False)
    h = make_product(pb, sysd, "fp64")
    psi = torch.as_tensor(sysd["psi"]).to("cuda")
    before = h.apply(psi)

    V = sysd["V"].copy()
    V[17] = np.nan
    with pytest.raises(pb.InqbError) as e:
        h.set_scalar_potential(V)
    assert e.value.status == 5
    with pytest.raises(pb.InqbError) as e:
        h.set_vector_potential_cov(np.array([0.0, np.inf, 0.0]))
    assert e.value.status == 5
    x = psi.clone()
    with pytest.raises(pb.InqbError) as e:
        h.kick_(x, [np.nan, 0.0, 0.0])
    assert e.value.status == 5
    assert torch.equal(x, psi)
    with pytest.raises(pb.InqbError) as e:
        h.crank_nicolson_step_(x, float("nan"), np.zeros(3), np.zeros(3))
    assert e.value.status == 1
    assert torch.equal(x, psi)

    after = h.apply(psi)
    assert torch.equal(after, before)
