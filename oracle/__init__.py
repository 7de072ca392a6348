"""ORACLE — test infrastructure only.

ctypes wrapper around ``oracle/liboracle.so``, the CPU FP64 restatement of INQ's
Kohn-Sham Hamiltonian hot path (``oracle/oracle.cpp`` lists, for every routine,
the reference file and lines it follows).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module; the product (``inq-wannier-fork_b200``) never does.

Parity: pinned against the golden values of the reference's unit tests (see
``tests/test_oracle_golden.py``); the projector tables and the ETRS/CN steps are
parity-unpinned conventions because the reference's own tests for them are empty
or need the absent pseudopod library.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++, OpenMP)."""
    src = os.path.join(_HERE, "oracle.cpp")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [_dp, _ip]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_volume_element.restype = ctypes.c_double
        L.orc_volume_element.argtypes = [ctypes.c_void_p]
        L.orc_set_potential.argtypes = [ctypes.c_void_p, _dp]
        L.orc_set_vector_potential_cov.argtypes = [ctypes.c_void_p, _dp]
        L.orc_cart_to_cov.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_set_fourier_mask.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_sphere.restype = ctypes.c_int
        L.orc_sphere.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, _ip, _fp, _fp]
        L.orc_gaussian_beta.argtypes = [ctypes.c_void_p, ctypes.c_int, _fp, _fp, ctypes.c_double, _dp]
        L.orc_set_projectors.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         _ip, _ip, _fp, _dp, _dp]
        L.orc_apply_h.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_fft3d.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.orc_exponential_in_place.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_double, _dp, ctypes.c_int]
        L.orc_etrs_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.orc_density.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.orc_dipole.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_band_energies.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.orc_crank_nicolson_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp,
                                              ctypes.c_int, ctypes.c_double, _ip, _dp]
        L.orc_rvectors.argtypes = [ctypes.c_void_p, _dp]
        L.orc_orthonormalize.restype = ctypes.c_int
        L.orc_orthonormalize.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.orc_poisson.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_lda_functional.restype = ctypes.c_double
        L.orc_lda_functional.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_ks_potential.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.orc_integral_sum_absdiff.restype = ctypes.c_double
        L.orc_integral_sum_absdiff.argtypes = [ctypes.c_void_p, ctypes.c_long, _dp, _dp]
        L.orc_etrs_scf_step.restype = ctypes.c_int
        L.orc_etrs_scf_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp, _dp,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp]
        L.orc_least_squares_sym.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_broyden_create.restype = ctypes.c_void_p
        L.orc_broyden_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_long]
        L.orc_broyden_destroy.argtypes = [ctypes.c_void_p]
        L.orc_broyden_mix.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.orc_density_normalize.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double]
        L.orc_crank_nicolson_scf_step.restype = ctypes.c_int
        L.orc_crank_nicolson_scf_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, _dp, _dp,
                                                  ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_double, _dp, _dp, _dp, _dp]
        L.orc_mlwf_matrices.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_jade.restype = ctypes.c_int
        L.orc_jade.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp]
        L.orc_mlwf_rotate.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_kick.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f(a):
    return a.ctypes.data_as(_fp)


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


class System:
    """FP64 Hamiltonian state on one cell/grid (mirrors ks_hamiltonian's members)."""

    def __init__(self, lattice, nr):
        self.lattice = np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).reshape(3, 3))
        self.nr = np.ascontiguousarray(np.asarray(nr, dtype=np.int32).reshape(3))
        self.N = int(np.prod(self.nr))
        self._h = lib().orc_create(_d(self.lattice), _i(self.nr))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.orc_destroy(h)
            self._h = None

    @property
    def volume_element(self) -> float:
        return float(lib().orc_volume_element(self._h))

    def set_potential(self, V):
        V = np.ascontiguousarray(V, dtype=np.float64).reshape(self.N)
        lib().orc_set_potential(self._h, _d(V))

    def set_vector_potential_cov(self, kA):
        kA = np.ascontiguousarray(kA, dtype=np.float64).reshape(3)
        lib().orc_set_vector_potential_cov(self._h, _d(kA))

    def set_fourier_mask(self, enable=True):
        lib().orc_set_fourier_mask(self._h, int(bool(enable)))

    def cart_to_cov(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(3)
        out = np.zeros(3)
        lib().orc_cart_to_cov(self._h, _d(v), _d(out))
        return out

    def sphere(self, center, radius):
        c = np.ascontiguousarray(center, dtype=np.float64).reshape(3)
        n = lib().orc_sphere(self._h, _d(c), float(radius), None, None, None)
        coords = np.zeros((n, 3), np.int32)
        dist = np.zeros(n, np.float32)
        relpos = np.zeros((n, 3), np.float32)
        lib().orc_sphere(self._h, _d(c), float(radius), _i(coords), _f(dist), _f(relpos))
        return coords, dist, relpos

    def gaussian_beta(self, dist, relpos, sigma=1.0):
        n = len(dist)
        dist = np.ascontiguousarray(dist, np.float32)
        relpos = np.ascontiguousarray(relpos, np.float32)
        beta = np.zeros((4, n))
        lib().orc_gaussian_beta(self._h, n, _f(dist), _f(relpos), float(sigma), _d(beta))
        return beta

    def build_gaussian_kb(self, positions, radius=3.0, sigma=1.0, ekb_s=1.5, ekb_p=-0.7):
        """Per-atom spheres + beta tables padded to the largest sphere (projector_all layout)."""
        spheres = [self.sphere(p, radius) for p in np.asarray(positions, float).reshape(-1, 3)]
        nproj = len(spheres)
        smax = max([len(s[1]) for s in spheres] + [0])
        counts = np.array([len(s[1]) for s in spheres], np.int32)
        coords = -np.ones((nproj, smax, 3), np.int32)
        relpos = np.zeros((nproj, smax, 3), np.float32)
        beta = np.zeros((nproj, 4, smax))
        for a, (c, d, r) in enumerate(spheres):
            n = len(d)
            coords[a, :n] = c
            relpos[a, :n] = r
            beta[a, :, :n] = self.gaussian_beta(d, r, sigma)
        coeff = np.tile(np.array([ekb_s, ekb_p, ekb_p, ekb_p]), (nproj, 1))
        return dict(counts=counts, coords=coords, relpos=relpos, beta=beta, coeff=coeff, smax=smax, L=4)

    def set_projectors(self, kb):
        nproj = len(kb["counts"])
        self._kb = {k: np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v for k, v in kb.items()}
        k = self._kb
        lib().orc_set_projectors(self._h, nproj, int(k["L"]), int(k["smax"]),
                                 _i(k["counts"].astype(np.int32)), _i(k["coords"].astype(np.int32)),
                                 _f(k["relpos"].astype(np.float32)), _d(k["beta"].astype(np.float64)),
                                 _d(k["coeff"].astype(np.float64)))

    def _psi(self, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        assert psi.ndim == 2 and psi.shape[0] == self.N
        return psi

    def apply_h(self, psi):
        psi = self._psi(psi)
        out = np.zeros_like(psi)
        lib().orc_apply_h(self._h, psi.shape[1], _d(psi.view(np.float64)), _d(out.view(np.float64)))
        return out

    def fft3d(self, psi, sign=-1, normalize=False):
        psi = self._psi(psi)
        out = np.zeros_like(psi)
        lib().orc_fft3d(self._h, psi.shape[1], _d(psi.view(np.float64)), _d(out.view(np.float64)),
                        int(sign), int(bool(normalize)))
        return out

    def exponential(self, factor, psi, order=4):
        out = self._psi(psi).copy()
        lib().orc_exponential_in_place(self._h, out.shape[1], float(np.real(factor)), float(np.imag(factor)),
                                       _d(out.view(np.float64)), int(order))
        return out

    def etrs_step(self, psi, dt, kA_t, kA_tdt):
        out = self._psi(psi).copy()
        a = np.ascontiguousarray(kA_t, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt, np.float64).reshape(3)
        lib().orc_etrs_step(self._h, out.shape[1], float(dt), _d(a), _d(b), _d(out.view(np.float64)))
        return out

    def crank_nicolson_step(self, psi, dt, kA_t, kA_tdt, max_sweeps=300, tol=1e-10):
        """(new orbitals, sweeps run, last residual)"""
        out = self._psi(psi).copy()
        a = np.ascontiguousarray(kA_t, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt, np.float64).reshape(3)
        k = ctypes.c_int(0)
        r = ctypes.c_double(0.0)
        lib().orc_crank_nicolson_step(self._h, out.shape[1], float(dt), _d(a), _d(b), _d(out.view(np.float64)),
                                      int(max_sweeps), float(tol), ctypes.byref(k), ctypes.byref(r))
        return out, k.value, r.value

    def density(self, psi, occ):
        psi = self._psi(psi)
        occ = np.ascontiguousarray(occ, np.float64).reshape(psi.shape[1])
        rho = np.zeros(self.N)
        lib().orc_density(self._h, psi.shape[1], _d(psi.view(np.float64)), _d(occ), _d(rho))
        return rho

    def dipole(self, rho):
        rho = np.ascontiguousarray(rho, np.float64).reshape(self.N)
        out = np.zeros(3)
        lib().orc_dipole(self._h, _d(rho), _d(out))
        return out

    def band_energies(self, psi, hpsi):
        psi = self._psi(psi)
        hpsi = self._psi(hpsi)
        eps = np.zeros(psi.shape[1])
        lib().orc_band_energies(self._h, psi.shape[1], _d(psi.view(np.float64)), _d(hpsi.view(np.float64)), _d(eps))
        return eps

    def rvectors(self):
        out = np.zeros((self.N, 3))
        lib().orc_rvectors(self._h, _d(out))
        return out

    def orthonormalize(self, psi):
        out = self._psi(psi).copy()
        info = lib().orc_orthonormalize(self._h, out.shape[1], _d(out.view(np.float64)))
        if info != 0:
            raise ArithmeticError(f"overlap matrix not positive definite at pivot {info - 1}")
        return out

    # ---- density -> potential (self_consistency.hpp:89-160)

    def poisson(self, fields):
        """solvers::poisson (periodic) of complex fields [N] or [N][M]."""
        f = np.asarray(fields, dtype=np.complex128)
        shape = f.shape
        f = np.ascontiguousarray(f.reshape(self.N, -1))
        out = np.zeros_like(f)
        lib().orc_poisson(self._h, f.shape[1], _d(f.view(np.float64)), _d(out.view(np.float64)))
        return out.reshape(shape)

    def lda_functional(self, func, rho):
        """(v, efunc) of XC_LDA_X (func 1) or XC_LDA_C_PZ (func 9); rho [N] or [N][2]."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        nspin = 1 if rho.ndim == 1 else rho.shape[1]
        if rho.shape[0] != self.N or nspin not in (1, 2):
            raise ValueError("rho must be [N] or [N][2]")
        v = np.zeros_like(rho)
        e = lib().orc_lda_functional(self._h, int(func), int(nspin), _d(rho), _d(v))
        return v, e

    def ks_potential(self, rho, vion, theory):
        """update_hamiltonian: sets V = vion + V_H + V_xc; returns (V, energies
        {external, hartree, xc, nvxc}).  theory 0 none, 1 Hartree, 2 LDA."""
        rho = np.ascontiguousarray(rho, np.float64).reshape(self.N)
        vion = np.ascontiguousarray(vion, np.float64).reshape(self.N)
        V = np.zeros(self.N)
        en = np.zeros(4)
        lib().orc_ks_potential(self._h, _d(rho), _d(vion), int(theory), _d(V), _d(en))
        return V, en

    def integral_sum_absdiff(self, a, b):
        a = np.ascontiguousarray(a, np.float64).ravel()
        b = np.ascontiguousarray(b, np.float64).ravel()
        return lib().orc_integral_sum_absdiff(self._h, a.size, _d(a), _d(b))

    def kick(self, psi, kick_cart):
        """perturbations::kick::zero_step, length gauge: psi exp(-i kick . r)."""
        out = self._psi(psi).copy()
        k = np.ascontiguousarray(kick_cart, np.float64).reshape(3)
        lib().orc_kick(self._h, out.shape[1], _d(out.view(np.float64)), _d(k))
        return out

    # ---- TD-MLWF (wannier/tdmlwf_trans.hpp)

    def mlwf_matrices(self, psi):
        """tdmlwf_trans::update: the six [M][M] matrices of the normalised states."""
        psi = self._psi(psi)
        M = psi.shape[1]
        a = np.zeros((6, M, M), np.complex128)
        lib().orc_mlwf_matrices(self._h, M, _d(psi.view(np.float64)), _d(a.view(np.float64)))
        return a

    def mlwf_rotate(self, psi, u):
        """apply_transform: psi u^H (operations::rotate)."""
        out = self._psi(psi).copy()
        u = np.ascontiguousarray(u, np.complex128)
        lib().orc_mlwf_rotate(self._h, out.shape[1], _d(out.view(np.float64)), _d(u.view(np.float64)))
        return out

    def etrs_scf_step(self, psi, rho, dt, kA_t, kA_tdt, occ, vion, theory, nscf=5, threshold=5e-5):
        """ETRS with its SCF loop (etrs.hpp:22-82).  The potential must already be the
        Kohn-Sham potential of rho.  Returns (psi, rho, scf iterations, energies)."""
        out = self._psi(psi).copy()
        r = np.ascontiguousarray(rho, np.float64).reshape(self.N).copy()
        a = np.ascontiguousarray(kA_t, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt, np.float64).reshape(3)
        occ = np.ascontiguousarray(occ, np.float64).reshape(out.shape[1])
        vion = np.ascontiguousarray(vion, np.float64).reshape(self.N)
        en = np.zeros(4)
        it = lib().orc_etrs_scf_step(self._h, out.shape[1], float(dt), _d(a), _d(b), _d(occ), _d(vion),
                                     int(theory), int(nscf), float(threshold), _d(out.view(np.float64)),
                                     _d(r), _d(en))
        return out, r, it, en


    def density_normalize(self, rho, total):
        """observables::density::normalize (density.hpp:100-111): rho * total / (dV sum rho)."""
        r = np.ascontiguousarray(rho, np.float64).reshape(self.N).copy()
        lib().orc_density_normalize(self._h, _d(r), float(total))
        return r

    def crank_nicolson_scf_step(self, psi, rho, dt, kA_t, kA_tdt, occ, vion, theory, nelec=None, max_iter=300,
                                dens_tol=1e-5):
        """Crank-Nicolson with its self-consistency loop and Broyden density mixing
        (crank_nicolson.hpp:41-114).  The potential must already be the Kohn-Sham
        potential of rho.  nelec defaults to sum(occ).  Returns (psi, rho, iterations,
        energies, last solver residual)."""
        out = self._psi(psi).copy()
        r = np.ascontiguousarray(rho, np.float64).reshape(self.N).copy()
        a = np.ascontiguousarray(kA_t, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt, np.float64).reshape(3)
        occ = np.ascontiguousarray(occ, np.float64).reshape(out.shape[1])
        vion = np.ascontiguousarray(vion, np.float64).reshape(self.N)
        nelec = float(occ.sum()) if nelec is None else float(nelec)
        en = np.zeros(4)
        res = np.zeros(1)
        it = lib().orc_crank_nicolson_scf_step(self._h, out.shape[1], float(dt), _d(a), _d(b), _d(occ), nelec,
                                               _d(vion), int(theory), int(max_iter), float(dens_tol),
                                               _d(out.view(np.float64)), _d(r), _d(en), _d(res))
        return out, r, it, en, float(res[0])


def least_squares_sym(a, b):
    """solvers::least_squares (least_squares.hpp:27-54, dgelsd with rcond -1) for a
    symmetric matrix: the minimum-norm least-squares solution of a x = b."""
    a = np.ascontiguousarray(a, np.float64).copy()
    n = a.shape[0]
    if a.shape != (n, n):
        raise ValueError("a must be square")
    x = np.ascontiguousarray(b, np.float64).reshape(n).copy()
    lib().orc_least_squares_sym(n, _d(a), _d(x))
    return x


class Broyden:
    """mixers::broyden (src/mixers/broyden.hpp:26-160) on a real vector of dim values:
    mix(vin, vout) returns the new input."""

    def __init__(self, steps, mix, dim):
        self.dim = int(dim)
        self._h = lib().orc_broyden_create(int(steps), float(mix), self.dim)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_broyden_destroy(self._h)
            self._h = None

    def mix(self, vin, vout):
        vin = np.ascontiguousarray(vin, np.float64).reshape(self.dim).copy()
        vout = np.ascontiguousarray(vout, np.float64).reshape(self.dim)
        lib().orc_broyden_mix(self._h, _d(vin), _d(vout))
        return vin


# ---- checkpoint layout (operations/io.hpp:42-177, systems/electrons.hpp:323-375)

def num_to_str(n: int) -> str:
    """utils::num_to_str (src/utils/num_str.hpp:20-24): "%010ld" into an 11-byte buffer."""
    return ("%010d" % int(n))[:10]


def save_orbitals_layout(dirname, psi, occ=None, kpin=0, first_state=0):
    """The files systems::electrons::save writes for one k-point block: one raw
    complex128 file per state (io::save(orbital_set), spinor 0) and the occupations
    array written at offset first_state (io::save(array))."""
    psi = np.asarray(psi)
    kdir = os.path.join(dirname, "kpin" + num_to_str(kpin))
    os.makedirs(os.path.join(kdir, "states"), exist_ok=True)
    for j in range(psi.shape[1]):
        name = num_to_str(first_state + j) + "_" + num_to_str(0)
        np.ascontiguousarray(psi[:, j], dtype=np.complex128).tofile(os.path.join(kdir, "states", name))
    if occ is not None:
        os.makedirs(os.path.join(kdir, "occupations"), exist_ok=True)
        path = os.path.join(kdir, "occupations", "array")
        mode = "r+b" if os.path.exists(path) else "wb"
        with open(path, mode) as f:
            f.seek(8 * first_state)
            f.write(np.ascontiguousarray(occ, dtype=np.float64).tobytes())


def load_orbitals_layout(dirname, N, M, kpin=0, first_state=0):
    """(psi [N, M] complex128, occupations [M]) read back from that layout."""
    kdir = os.path.join(dirname, "kpin" + num_to_str(kpin))
    psi = np.zeros((N, M), np.complex128)
    for j in range(M):
        name = num_to_str(first_state + j) + "_" + num_to_str(0)
        psi[:, j] = np.fromfile(os.path.join(kdir, "states", name), dtype=np.complex128, count=N)
    occ = np.fromfile(os.path.join(kdir, "occupations", "array"), dtype=np.float64)[first_state:first_state + M]
    return psi, occ


# ---- TD-MLWF (wannier/jade_complex.hpp, tdmlwf_trans.hpp:196-330)

def jade(a, maxsweep=100, tol=1e-8):
    """jade_complex: (a rotated, u, adiag, sweeps) for a [6][M][M] complex."""
    a = np.ascontiguousarray(a, np.complex128).copy()
    M = a.shape[1]
    u = np.zeros((M, M), np.complex128)
    adiag = np.zeros((6, M), np.complex128)
    sw = lib().orc_jade(int(maxsweep), float(tol), M, _d(a.view(np.float64)), _d(u.view(np.float64)),
                        _d(adiag.view(np.float64)))
    return a, u, adiag, sw


def mlwf_center(adiag, i, lattice):
    """tdmlwf_trans::center (tdmlwf_trans.hpp:196-220): t_d = atan2(Re s_d, Re c_d) / 2 pi,
    r = L t with L's rows the lattice vectors, as the reference writes it."""
    L = np.asarray(lattice, float).reshape(3, 3)
    t = [np.arctan2(adiag[2 * d + 1][i].real, adiag[2 * d][i].real) / (2 * np.pi) for d in range(3)]
    return np.array([t[0] * L[0, 0] + t[1] * L[0, 1] + t[2] * L[0, 2],
                     t[0] * L[1, 0] + t[1] * L[1, 1] + t[2] * L[1, 2],
                     t[0] * L[2, 0] + t[1] * L[2, 1] + t[2] * L[2, 2]])


def mlwf_spread(adiag, i, lattice):
    """tdmlwf_trans::spread (tdmlwf_trans.hpp:286-312): sqrt(sum_d (1 - |c_d|^2 - |s_d|^2) / |b_d|^2)."""
    L = np.asarray(lattice, float).reshape(3, 3)
    B = 2 * np.pi * np.linalg.inv(L).T  # rows: reciprocal vectors (cell.hpp:50-52)
    s2 = 0.0
    for d in range(3):
        c, s = adiag[2 * d][i], adiag[2 * d + 1][i]
        s2 += (1.0 - abs(c) ** 2 - abs(s) ** 2) / (B[d] @ B[d])
    return np.sqrt(s2)
