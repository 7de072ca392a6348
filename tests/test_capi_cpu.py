"""CPU checks of the C ABI: the library loads, exports every symbol the header
declares, and its setup helpers (no GPU needed) agree bit for bit with the oracle."""
import ctypes
import re

import numpy as np
import pytest

from pinq_b200 import systems


def _declared_symbols():
    from pinq_b200 import _lib

    text = open(_lib.HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(inqb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(pb):
    lib = pb.lib()
    names = _declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(pb):
    from pinq_b200 import _lib

    assert set(_declared_symbols()) == set(_lib.SIGNATURES)


def test_status_strings(pb):
    lib = pb.lib()
    assert lib.inqb_version() >= 1
    assert lib.inqb_status_string(0) == b"ok"
    assert lib.inqb_status_string(6) == b"matrix not positive definite"
    assert lib.inqb_status_string(8) == b"checkpoint file missing, short or unwritable"


def test_grid_support_table(pb):
    """Every length of the FFT size table as a cubic grid, plus the compiled
    orthorhombic and tetragonal grids; lengths outside the table are not compiled."""
    for n in (12, 16, 18, 20, 24, 30, 32, 36, 40, 48, 60, 64, 72, 80, 96, 128, 144):
        assert pb.grid_supported((n, n, n), "fp64") and pb.grid_supported((n, n, n), "mixed"), n
    for nr in ((18, 24, 20), (36, 48, 60), (24, 24, 48), (32, 32, 48), (64, 64, 96)):
        assert pb.grid_supported(nr, "fp64") and pb.grid_supported(nr, "mixed"), nr
    assert not pb.grid_supported((17, 17, 17), "fp64")
    assert not pb.grid_supported((36, 60, 48), "mixed")


def test_context_needs_a_gpu_or_reports_an_error(pb):
    """Without a device the context constructor fails with a status, never crashes."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pb.InqbError) as e:
        pb.KSHamiltonian(np.eye(3) * 10.0, (20, 20, 20))
    assert e.value.status == 3  # INQB_ERR_CUDA


def test_unsupported_grid_is_rejected(pb):
    with pytest.raises(pb.InqbError) as e:
        pb.KSHamiltonian(np.eye(3) * 10.0, (17, 17, 17))
    assert e.value.status == 2  # INQB_ERR_UNSUPPORTED


@pytest.mark.parametrize("case", ["cfg0", "fcc", "small_cell", "corner"])
def test_sphere_and_beta_match_oracle_bitwise(pb, oracle_mod, case):
    if case == "cfg0":
        lat, nr, centers = systems.cubic(10.26), (32, 32, 32), list(systems.diamond_positions(10.26))
    elif case == "fcc":
        ll = 5.89
        lat, nr, centers = np.array([[0, ll, ll], [ll, 0, ll], [ll, ll, 0.0]]), (17, 17, 17), [(1.0, 2.0, 3.0)]
    elif case == "small_cell":  # sphere wider than half the cell: many replicas
        lat, nr, centers = systems.cubic(5.0), (16, 16, 16), [(0.3, -0.2, 0.1)]
    else:
        lat, nr, centers = systems.cubic(10.0), (20, 20, 20), [(-5.0, -5.0, -5.0), (5.0, 5.0, 5.0)]
    o = oracle_mod.System(lat, nr)
    for c in centers:
        c = np.asarray(c, float)
        c1, d1, r1 = o.sphere(c, 3.0)
        c2, d2, r2 = pb.sphere(lat, nr, c, 3.0)
        assert len(d1) == len(d2) > 0
        assert np.array_equal(c1, c2) and np.array_equal(d1, d2) and np.array_equal(r1, r2)
        assert np.array_equal(o.gaussian_beta(d1, r1), pb.gaussian_beta(lat, d2, r2))


def test_sphere_golden_257_through_the_library(pb):
    """spherical_grid.hpp:264-376 golden value through the product's setup code."""
    for c in [(0, 0, 0), (-5, 0, 0), (5, 5, 5), (2.5, 2.5, 2.5)]:
        assert len(pb.sphere(np.eye(3) * 10.0, (20, 20, 20), c, 2.0)[1]) == 257


def test_setup_argument_errors(pb):
    from pinq_b200 import _lib

    lat = np.ascontiguousarray(np.eye(3).reshape(9) * 10.0)
    nr = np.array([20, 20, 20], np.int32)
    c = np.zeros(3)
    n = ctypes.c_int(0)
    assert pb.lib().inqb_sphere_size(_lib.dptr(lat), _lib.iptr(nr), _lib.dptr(c), -1.0, ctypes.byref(n)) == 1
    bad = np.array([20, 0, 20], np.int32)
    assert pb.lib().inqb_sphere_size(_lib.dptr(lat), _lib.iptr(bad), _lib.dptr(c), 2.0, ctypes.byref(n)) == 1
    assert b"grid" in pb.lib().inqb_last_error()


def test_new_entry_points_reject_a_null_context(pb):
    """The density -> potential, checkpoint, TD-MLWF and kick entry points check their
    context before touching a device."""
    lib = pb.lib()
    three = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    assert lib.inqb_poisson(None, None, None, 1, 1, None) == 1
    assert lib.inqb_ks_potential(None, None, None, 2, None, None) == 1
    assert lib.inqb_set_density_reduce(None, None, None) == 1
    assert lib.inqb_save_orbitals(None, b"x", 0, None, 1, 1, 0, None, None) == 1
    assert lib.inqb_load_density(None, b"x", None, None) == 1
    assert lib.inqb_mlwf_step(None, None, 1, 1, 100, 1e-8, None, None, None, None) == 1
    assert lib.inqb_jade(None, 2, None, None, None, 100, 1e-8, None, None) == 1
    assert lib.inqb_kick(None, None, 1, 1, three, None) == 1
    assert lib.inqb_crank_nicolson_scf_step(None, None, 1, 1, 0.05, three, three, None, 2.0, None, None, 2, 300,
                                            1e-5, None, None, None, None) == 1
    assert b"null context" in lib.inqb_last_error()
