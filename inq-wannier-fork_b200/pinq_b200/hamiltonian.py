"""Python face of libinqb200, mirroring INQ's ``hamiltonian::ks_hamiltonian``.

Device memory comes from torch (CUDA tensors shaped ``[N, M]``, orbital index
fastest, as INQ's ``orbital_set``); every computation runs in the library's CUDA
kernels through the C ABI.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import FP64, MIXED, call, dptr, fptr, iptr


def _precision(p) -> int:
    if p in (FP64, "fp64", "double", torch.complex128):
        return FP64
    if p in (MIXED, "mixed", "fp32", torch.complex64):
        return MIXED
    raise ValueError(f"unknown precision {p!r}")


def _lattice(lattice) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).reshape(9))


# ------------------------------------------------------------------ setup helpers (no GPU)
def sphere(lattice, nr, center, radius):
    """Atom sphere of INQ's spherical_grid: (coords [n,3] int32, distance [n] float32, relpos [n,3] float32)."""
    lat = _lattice(lattice)
    n = np.ascontiguousarray(np.asarray(nr, dtype=np.int32).reshape(3))
    c = np.ascontiguousarray(np.asarray(center, dtype=np.float64).reshape(3))
    cnt = ctypes.c_int(0)
    call("inqb_sphere_size", dptr(lat), iptr(n), dptr(c), float(radius), ctypes.byref(cnt))
    npts = cnt.value
    coords = np.zeros((npts, 3), np.int32)
    dist = np.zeros(npts, np.float32)
    rel = np.zeros((npts, 3), np.float32)
    if npts:
        call("inqb_sphere_points", dptr(lat), iptr(n), dptr(c), float(radius), npts, iptr(coords), fptr(dist),
             fptr(rel))
    return coords, dist, rel


def gaussian_beta(lattice, dist, relpos, sigma=1.0):
    """KB tables beta[4][n] for (s, p-1, p0, p+1) Gaussian projectors."""
    lat = _lattice(lattice)
    dist = np.ascontiguousarray(dist, np.float32)
    relpos = np.ascontiguousarray(relpos, np.float32)
    beta = np.zeros((4, len(dist)))
    if len(dist):
        call("inqb_gaussian_kb_beta", dptr(lat), len(dist), fptr(dist), fptr(relpos), float(sigma), dptr(beta))
    return beta


def build_gaussian_kb(lattice, nr, positions, radius=3.0, sigma=1.0, ekb_s=1.5, ekb_p=-0.7):
    """projector_all-style tables for Gaussian s+p KB projectors on every atom."""
    spheres = [sphere(lattice, nr, p, radius) for p in np.asarray(positions, float).reshape(-1, 3)]
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
        beta[a, :, :n] = gaussian_beta(lattice, d, r, sigma)
    coeff = np.tile(np.array([ekb_s, ekb_p, ekb_p, ekb_p]), (nproj, 1))
    return dict(counts=counts, coords=coords, relpos=relpos, beta=beta, coeff=coeff, smax=smax, L=4)


def grid_supported(nr, precision="fp64") -> bool:
    return bool(_lib.lib().inqb_grid_supported(int(nr[0]), int(nr[1]), int(nr[2]), _precision(precision)))


# ------------------------------------------------------------------ the Hamiltonian
class _DeviceDoubles:
    """n FP64 values of device memory at ptr, exposed through __cuda_array_interface__
    so torch.as_tensor makes a view of them (no copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "strides": None, "version": 3}


class KSHamiltonian:
    """H|psi> and propagators for one cell/grid on one GPU (drop-in for ks_hamiltonian)."""

    # INQ's exchange_operator::enabled(): |coefficient| > 1e-14 (exchange_operator.hpp:229-231)
    EXCHANGE_THRESHOLD = 1.0e-14

    def __init__(self, lattice, nr, precision="fp64", device: int = 0, exchange_coefficient: float = 0.0):
        """exchange_coefficient: the theory's exact-exchange fraction (ks_hamiltonian.hpp:80).
        Exact exchange is not provided, so only 0 is accepted (ValueError otherwise,
        before any device work); exchange_enabled is then False, as INQ's
        exchange().enabled() is for these theories."""
        if abs(float(exchange_coefficient)) > self.EXCHANGE_THRESHOLD:
            raise ValueError(f"exact exchange is not provided (exchange coefficient {exchange_coefficient}, "
                             "only 0 is supported)")
        self.exchange_enabled = False
        self.lattice = _lattice(lattice).reshape(3, 3).copy()
        self.nr = tuple(int(n) for n in nr)
        self.N = int(np.prod(self.nr))
        self.precision = _precision(precision)
        self.dtype = torch.complex128 if self.precision == FP64 else torch.complex64
        self.device = torch.device("cuda", device)
        h = ctypes.c_void_p()
        call("inqb_ctx_create", dptr(_lattice(lattice)), self.nr[0], self.nr[1], self.nr[2], self.precision,
             int(device), ctypes.byref(h))
        self._h = h
        self.state_version = 0  # bumped by every call that changes the Hamiltonian (see clone)

    def clone(self) -> "KSHamiltonian":
        """A second context with this one's state (potential as it is on the device,
        vector potential, mask, projectors, projection form, schedules) and its own
        workspace, for work on another CUDA stream beside this one."""
        other = KSHamiltonian.__new__(KSHamiltonian)
        other.lattice = self.lattice.copy()
        other.nr = self.nr
        other.N = self.N
        other.precision = self.precision
        other.dtype = self.dtype
        other.device = self.device
        other.exchange_enabled = False
        h = ctypes.c_void_p()
        call("inqb_ctx_clone", self._h, ctypes.byref(h))
        other._h = h
        other.state_version = 0
        return other

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().inqb_ctx_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state
    @property
    def volume_element(self) -> float:
        return float(_lib.lib().inqb_volume_element(self._h))

    def cart_to_cov(self, v):
        v = np.ascontiguousarray(v, np.float64).reshape(3)
        out = np.zeros(3)
        call("inqb_cart_to_cov", self._h, dptr(v), dptr(out))
        return out

    def set_scalar_potential(self, V):
        self.state_version += 1
        V = np.ascontiguousarray(torch.as_tensor(V).detach().cpu().numpy() if torch.is_tensor(V) else V,
                                 dtype=np.float64).reshape(self.N)
        call("inqb_set_local_potential", self._h, dptr(V))

    def set_vector_potential_cov(self, kA_cov):
        kA = np.ascontiguousarray(kA_cov, np.float64).reshape(3)
        call("inqb_set_vector_potential", self._h, dptr(kA))

    def set_uniform_vector_potential(self, A_cart, kpoint_cart=(0.0, 0.0, 0.0)):
        self.set_vector_potential_cov(self.cart_to_cov(np.asarray(A_cart, float) + np.asarray(kpoint_cart, float)))

    def set_fourier_sphere_mask(self, enable: bool = True):
        """INQ's zero_outside_sphere on the kinetic term (off by default, as in INQ)."""
        self.state_version += 1
        call("inqb_set_fourier_sphere_mask", self._h, int(bool(enable)))

    def set_projectors(self, kb):
        self.state_version += 1
        nproj = len(kb["counts"])
        counts = np.ascontiguousarray(kb["counts"], np.int32)
        coords = np.ascontiguousarray(kb["coords"], np.int32)
        relpos = np.ascontiguousarray(kb["relpos"], np.float32)
        beta = np.ascontiguousarray(kb["beta"], np.float64)
        coeff = np.ascontiguousarray(kb["coeff"], np.float64)
        call("inqb_set_projectors", self._h, nproj, int(kb["L"]), int(kb["smax"]), iptr(counts), iptr(coords),
             fptr(relpos), dptr(beta), dptr(coeff))

    def set_gaussian_projectors(self, positions, radius=3.0, sigma=1.0, ekb_s=1.5, ekb_p=-0.7):
        kb = build_gaussian_kb(self.lattice, self.nr, positions, radius, sigma, ekb_s, ekb_p)
        self.set_projectors(kb)
        return kb

    def autotune(self, M: int) -> tuple:
        """Time the launch schedules for M orbitals and keep the fastest; returns
        (ysplit, threads of the three passes)."""
        self.state_version += 1
        sched = (ctypes.c_int * 4)()
        call("inqb_autotune", self._h, int(M), self._stream(), sched)
        return tuple(sched)

    def set_schedule(self, M: int, schedule=None):
        """Use schedule (ysplit, t1, t2, t3) for M orbitals; None restores the default."""
        self.state_version += 1
        arr = None if schedule is None else (ctypes.c_int * 4)(*[int(v) for v in schedule])
        call("inqb_set_schedule", self._h, int(M), arr)

    def reserve(self, M: int):
        call("inqb_ctx_reserve", self._h, int(M))

    # -- helpers
    def _check(self, psi: torch.Tensor) -> torch.Tensor:
        if not torch.is_tensor(psi) or psi.device.type != "cuda":
            raise TypeError("orbitals must be a CUDA tensor")
        if psi.dtype != self.dtype:
            raise TypeError(f"orbitals must be {self.dtype} for this precision, got {psi.dtype}")
        if psi.dim() != 2 or psi.shape[0] != self.N or psi.stride(1) != 1:
            raise ValueError(f"orbitals must be [N={self.N}, M] with unit orbital stride")
        return psi

    @staticmethod
    def _stream():
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _out_like(self, psi: torch.Tensor, out: torch.Tensor | None) -> torch.Tensor:
        """An output block for a call that takes one leading dimension for its input
        and output: psi's shape and row stride (a new block when out is None)."""
        if out is None:
            return torch.empty((psi.shape[0], psi.stride(0)), dtype=psi.dtype, device=psi.device)[:, :psi.shape[1]]
        out = self._check(out)
        if out.shape != psi.shape or out.stride(0) != psi.stride(0):
            raise ValueError("out must have the shape and the leading dimension (row stride) of the input")
        return out

    def empty(self, M: int) -> torch.Tensor:
        return torch.empty((self.N, M), dtype=self.dtype, device=self.device)

    # -- operations
    def apply(self, psi: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """out = H psi  (ks_hamiltonian::operator(); out may be psi)."""
        psi = self._check(psi)
        out = self._out_like(psi, out)
        call("inqb_apply_h", self._h, psi.data_ptr(), out.data_ptr(), psi.shape[1], psi.stride(0), self._stream())
        return out

    __call__ = apply

    def apply_host(self, psi_host: np.ndarray | torch.Tensor, out: np.ndarray | torch.Tensor | None = None):
        """H psi on host memory (copies in and out inside the call)."""
        if torch.is_tensor(psi_host):
            src = psi_host
            if not src.is_contiguous() or (out is not None and (not out.is_contiguous() or out.shape != src.shape)):
                raise ValueError("host blocks must be contiguous [N, M] tensors of one shape")
            if out is None:
                out = torch.empty_like(src)
            call("inqb_apply_h_host", self._h, src.data_ptr(), out.data_ptr(), src.shape[1])
            return out
        src = np.ascontiguousarray(psi_host)
        if out is None:
            out = np.empty_like(src)
        call("inqb_apply_h_host", self._h, src.ctypes.data, out.ctypes.data, src.shape[1])
        return out

    def to_fourier(self, psi, out=None):
        psi = self._check(psi)
        out = self._out_like(psi, out)
        call("inqb_fft_forward", self._h, psi.data_ptr(), out.data_ptr(), psi.shape[1], psi.stride(0), self._stream())
        return out

    def to_real(self, psi, out=None):
        psi = self._check(psi)
        out = self._out_like(psi, out)
        call("inqb_fft_backward", self._h, psi.data_ptr(), out.data_ptr(), psi.shape[1], psi.stride(0), self._stream())
        return out

    def kick_(self, psi, kick_cart):
        """perturbations::kick::zero_step in the length gauge: psi *= exp(-i kick . r)."""
        psi = self._check(psi)
        k = np.ascontiguousarray(kick_cart, np.float64).reshape(3)
        call("inqb_kick", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), dptr(k), self._stream())
        return psi

    # -- density -> potential (self_consistency.hpp:89-160)
    def poisson(self, fields, out=None):
        """solvers::poisson (periodic cell) of complex fields [N, M] in the context
        precision: V(G) = 4 pi rho(G) / |G|^2, 0 at G = 0."""
        fields = self._check(fields)
        out = self._out_like(fields, out)
        call("inqb_poisson", self._h, fields.data_ptr(), out.data_ptr(), fields.shape[1], fields.stride(0),
             self._stream())
        return out

    def _fp64_field(self, x, name):
        if x is None:
            return None
        if x.dtype != torch.float64 or x.device.type != "cuda" or x.numel() != self.N or not x.is_contiguous():
            raise TypeError(f"{name} must be a contiguous FP64 CUDA tensor of N values")
        return x

    def ks_potential(self, rho, vion=None, theory=2, energies=True):
        """update_hamiltonian: the local potential becomes vion + V_H[rho] + v_xc[rho]
        (theory 0 none, 1 Hartree, 2 LDA).  Returns the energies {external, hartree,
        xc, nvxc} (synchronises) or None."""
        self.state_version += 1
        rho = self._fp64_field(rho, "rho")
        vion = self._fp64_field(vion, "vion")
        en = np.zeros(4) if energies else None
        call("inqb_ks_potential", self._h, rho.data_ptr(), vion.data_ptr() if vion is not None else None, int(theory),
             dptr(en) if en is not None else None, self._stream())
        return dict(zip(("external", "hartree", "xc", "nvxc"), en.tolist())) if en is not None else None

    def etrs_scf_step_(self, psi, rho, dt, kA_t_cov, kA_tdt_cov, occ, vion=None, theory=2, nscf=5, threshold=5e-5):
        """ETRS with the self-consistency loop of real_time::etrs, in place on psi and
        rho (the potential must be the Kohn-Sham potential of rho on entry).
        Returns (SCF iterations, energies of the last update)."""
        self.state_version += 1
        psi = self._check(psi)
        rho = self._fp64_field(rho, "rho")
        vion = self._fp64_field(vion, "vion")
        occ_t = torch.as_tensor(occ, dtype=torch.float64, device=self.device).contiguous()
        if occ_t.numel() != psi.shape[1]:
            raise ValueError("one occupation per orbital")
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        it = ctypes.c_int(0)
        en = np.zeros(4)
        cb = None
        reducer = getattr(self, "_density_reducer", None)
        if reducer is not None:
            def _reduce(ptr, n, user, _rho=rho):
                try:
                    reducer(_rho)
                    return 0
                except Exception:  # reported to the caller as the step's failure
                    return 1
            cb = _lib.DENSITY_REDUCE_FN(_reduce)
            call("inqb_set_density_reduce", self._h, ctypes.cast(cb, ctypes.c_void_p), None)
        try:
            call("inqb_etrs_scf_step", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt), dptr(a),
                 dptr(b), occ_t.data_ptr(), rho.data_ptr(), vion.data_ptr() if vion is not None else None,
                 int(theory), int(nscf), float(threshold), ctypes.byref(it), dptr(en), self._stream())
        finally:
            if cb is not None:
                call("inqb_set_density_reduce", self._h, None, None)
        return it.value, dict(zip(("external", "hartree", "xc", "nvxc"), en.tolist()))

    def crank_nicolson_scf_step_(self, psi, rho, dt, kA_t_cov, kA_tdt_cov, occ, vion=None, theory=2, max_iter=300,
                                 dens_tol=1e-5, num_electrons=None):
        """Crank-Nicolson with the self-consistency loop and Broyden density mixing of
        real_time::crank_nicolson, in place on psi and rho (the potential must be the
        Kohn-Sham potential of rho on entry).  num_electrons defaults to sum(occ); an
        orbital-sharded run passes the total over the ranks.  Returns (iterations,
        last solver residual, energies of the last update)."""
        self.state_version += 1
        psi = self._check(psi)
        rho = self._fp64_field(rho, "rho")
        vion = self._fp64_field(vion, "vion")
        occ_t = torch.as_tensor(occ, dtype=torch.float64, device=self.device).contiguous()
        if occ_t.numel() != psi.shape[1]:
            raise ValueError("one occupation per orbital")
        nelec = float(occ_t.sum().item()) if num_electrons is None else float(num_electrons)
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        it = ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        en = np.zeros(4)
        cb = self._install_density_reducer()
        try:
            call("inqb_crank_nicolson_scf_step", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt),
                 dptr(a), dptr(b), occ_t.data_ptr(), nelec, rho.data_ptr(),
                 vion.data_ptr() if vion is not None else None, int(theory), int(max_iter), float(dens_tol),
                 ctypes.byref(it), ctypes.byref(res), dptr(en), self._stream())
        finally:
            if cb is not None:
                call("inqb_set_density_reduce", self._h, None, None)
        return it.value, res.value, dict(zip(("external", "hartree", "xc", "nvxc"), en.tolist()))

    def _install_density_reducer(self):
        """Registers the reducer set by set_density_reducer (if any) as the library's
        density-reduce callback; returns the ctypes callback to keep alive, or None.
        The reducer gets an FP64 tensor view of the buffer the library just filled
        (the step's own density or its scratch copy), not a copy."""
        reducer = getattr(self, "_density_reducer", None)
        if reducer is None:
            return None
        device = self.device

        def _reduce(ptr, n, user):
            try:
                with torch.cuda.device(device):
                    view = torch.as_tensor(_DeviceDoubles(ptr, n), device=device)
                if view.data_ptr() != int(ptr):  # a copy would not reach the library's buffer
                    return 1
                reducer(view)
                return 0
            except Exception:  # reported to the caller as the step's failure
                return 1
        cb = _lib.DENSITY_REDUCE_FN(_reduce)
        call("inqb_set_density_reduce", self._h, ctypes.cast(cb, ctypes.c_void_p), None)
        return cb

    def set_density_reducer(self, reducer):
        """Orbital-sharded SCF: reducer(rho) must replace rho (an FP64 CUDA tensor) by
        its sum over the ranks before returning, e.g. parallel.density_reducer(group).
        None removes it."""
        self.state_version += 1
        self._density_reducer = reducer

    # -- checkpoints in INQ's restart layout (operations/io.hpp, systems/electrons.hpp)
    def save_orbitals(self, dirname, psi, occ=None, kpin=0, first_state=0):
        """Write states first_state.. of k-point block kpin (and the occupations)
        under the electrons directory dirname, as complex128 files."""
        psi = self._check(psi)
        o = None if occ is None else np.ascontiguousarray(occ, np.float64).reshape(psi.shape[1])
        call("inqb_save_orbitals", self._h, os.fsencode(dirname), int(kpin), psi.data_ptr(), psi.shape[1],
             psi.stride(0), int(first_state), dptr(o) if o is not None else None, self._stream())

    def load_orbitals(self, dirname, psi, kpin=0, first_state=0, with_occupations=True):
        """Fill psi [N, M] from the files; returns the occupations (or None).  Raises
        InqbError (status ERR_IO) when a file is missing or short."""
        psi = self._check(psi)
        o = np.zeros(psi.shape[1]) if with_occupations else None
        call("inqb_load_orbitals", self._h, os.fsencode(dirname), int(kpin), psi.data_ptr(), psi.shape[1],
             psi.stride(0), int(first_state), dptr(o) if o is not None else None, self._stream())
        return o

    def save_density(self, dirname, rho):
        rho = self._fp64_field(rho, "rho")
        call("inqb_save_density", self._h, os.fsencode(dirname), rho.data_ptr(), self._stream())

    def load_density(self, dirname, rho=None):
        rho = torch.empty(self.N, dtype=torch.float64, device=self.device) if rho is None else \
            self._fp64_field(rho, "rho")
        call("inqb_load_density", self._h, os.fsencode(dirname), rho.data_ptr(), self._stream())
        return rho

    # -- TD-MLWF (wannier/tdmlwf_trans.hpp, observables/mlwf_properties.hpp)
    def mlwf_step_(self, psi, maxsweep=100, tol=1e-8):
        """update + compute_transform + apply_transform: psi is rotated in place to the
        maximally localised gauge; returns (centres [M, 3], spreads [M], JADE sweeps)."""
        psi = self._check(psi)
        M = psi.shape[1]
        centres = np.zeros((M, 3))
        spreads = np.zeros(M)
        sw = ctypes.c_int(0)
        call("inqb_mlwf_step", self._h, psi.data_ptr(), M, psi.stride(0), int(maxsweep), float(tol), ctypes.byref(sw),
             dptr(centres), dptr(spreads), self._stream())
        return centres, spreads, sw.value

    def mlwf_matrices(self, psi):
        """The six [M, M] complex128 matrices of tdmlwf_trans::update (a CUDA tensor)."""
        psi = self._check(psi)
        M = psi.shape[1]
        a = torch.empty((6, M, M), dtype=torch.complex128, device=self.device)
        call("inqb_mlwf_matrices", self._h, psi.data_ptr(), M, psi.stride(0), a.data_ptr(), self._stream())
        return a

    def jade(self, a, maxsweep=100, tol=1e-8):
        """jade_complex on a [6, M, M] complex128 CUDA tensor (rotated in place);
        returns (u, adiag, sweeps)."""
        if a.dtype != torch.complex128 or a.device.type != "cuda" or not a.is_contiguous() or a.shape[0] != 6:
            raise TypeError("a must be a contiguous [6, M, M] complex128 CUDA tensor")
        M = a.shape[1]
        u = torch.empty((M, M), dtype=torch.complex128, device=self.device)
        adiag = torch.empty((6, M), dtype=torch.complex128, device=self.device)
        sw = ctypes.c_int(0)
        call("inqb_jade", self._h, M, a.data_ptr(), u.data_ptr(), adiag.data_ptr(), int(maxsweep), float(tol),
             ctypes.byref(sw), self._stream())
        return u, adiag, sw.value

    def mlwf_rotate_(self, psi, u):
        """psi <- psi u^H (operations::rotate) with u an [M, M] complex128 CUDA tensor."""
        psi = self._check(psi)
        u = u.contiguous()
        call("inqb_mlwf_rotate", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), u.data_ptr(), self._stream())
        return psi

    def exponential_(self, psi, factor, order=4):
        """psi <- sum_k (factor H)^k / k! psi (in place)."""
        psi = self._check(psi)
        f = complex(factor)
        call("inqb_exponential", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), f.real, f.imag, int(order),
             self._stream())
        return psi

    def etrs_step_(self, psi, dt, kA_t_cov, kA_tdt_cov):
        psi = self._check(psi)
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        call("inqb_etrs_step", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt), dptr(a), dptr(b),
             self._stream())
        return psi

    def crank_nicolson_step_(self, psi, dt, kA_t_cov, kA_tdt_cov, max_sweeps=300, tol=1e-10):
        """One Crank-Nicolson step in place; returns (sweeps run, last residual)."""
        psi = self._check(psi)
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        k = ctypes.c_int(0)
        r = ctypes.c_double(0.0)
        call("inqb_crank_nicolson_step", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt), dptr(a),
             dptr(b), int(max_sweeps), float(tol), ctypes.byref(k), ctypes.byref(r), self._stream())
        return k.value, r.value

    def etrs_step_powers_(self, psi, dt, kA_t_cov, kA_tdt_cov, powers):
        """One ETRS step in place that also writes what the adjoint step reads (the
        Taylor powers and their forward coefficients) into `powers`, one row of
        powers_buffer(nsteps, M)."""
        psi = self._check(psi)
        self._check_powers(powers, psi.shape[1])
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        call("inqb_etrs_step_powers", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt), dptr(a),
             dptr(b), powers.data_ptr(), self._stream())
        return psi

    def etrs_step_terms_(self, psi, dt, kA_t_cov, kA_tdt_cov):
        """The step of etrs_step_powers_ keeping nothing: the same orbitals bit for bit."""
        psi = self._check(psi)
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        call("inqb_etrs_step_terms", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), float(dt), dptr(a),
             dptr(b), self._stream())
        return psi

    def etrs_adjoint_step_(self, lam, dt, kA_t_cov, kA_tdt_cov, powers, gV, gA_t, gA_tdt):
        """Reverse of one ETRS step: lam <- U^dagger lam and the V / A gradients
        accumulated into gV [N] and gA_t, gA_tdt [3] (FP64 CUDA tensors)."""
        lam = self._check(lam)
        self._check_powers(powers, lam.shape[1])
        for g, n in ((gV, self.N), (gA_t, 3), (gA_tdt, 3)):
            if g.dtype != torch.float64 or g.device.type != "cuda" or g.numel() < n or not g.is_contiguous():
                raise TypeError("gradients must be contiguous FP64 CUDA tensors")
        a = np.ascontiguousarray(kA_t_cov, np.float64).reshape(3)
        b = np.ascontiguousarray(kA_tdt_cov, np.float64).reshape(3)
        call("inqb_etrs_adjoint_step", self._h, lam.data_ptr(), lam.shape[1], lam.stride(0), float(dt), dptr(a),
             dptr(b), powers.data_ptr(), gV.data_ptr(), gA_t.data_ptr(), gA_tdt.data_ptr(), self._stream())
        return lam

    def powers_buffer(self, nsteps: int, M: int) -> torch.Tensor:
        """Storage for nsteps steps of etrs_step_powers_ ([nsteps, per-step elements];
        pass row n to the step and to its adjoint)."""
        nbytes = ctypes.c_size_t(0)
        call("inqb_etrs_powers_size", self._h, int(M), ctypes.byref(nbytes))
        esz = 16 if self.dtype == torch.complex128 else 8
        return torch.empty((int(nsteps), nbytes.value // esz), dtype=self.dtype, device=self.device)

    def _check_powers(self, powers, M):
        nbytes = ctypes.c_size_t(0)
        call("inqb_etrs_powers_size", self._h, int(M), ctypes.byref(nbytes))
        esz = 16 if self.dtype == torch.complex128 else 8
        if (not torch.is_tensor(powers) or powers.device.type != "cuda" or powers.dtype != self.dtype
                or powers.numel() * esz != nbytes.value or not powers.is_contiguous()
                or powers.data_ptr() % 16 != 0):
            raise ValueError("powers must be one row of powers_buffer(nsteps, M)")

    def density(self, psi, occ) -> torch.Tensor:
        psi = self._check(psi)
        occ_t = torch.as_tensor(occ, dtype=torch.float64, device=self.device).contiguous()
        rho = torch.empty(self.N, dtype=torch.float64, device=self.device)
        call("inqb_density", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), occ_t.data_ptr(), rho.data_ptr(),
             self._stream())
        return rho

    def dipole(self, rho: torch.Tensor) -> np.ndarray:
        rho = rho.contiguous()
        out = np.zeros(3)
        call("inqb_dipole", self._h, rho.data_ptr(), dptr(out), self._stream())
        return out

    # -- adjoint building blocks
    def axpby_(self, a, x, b, y):
        """y <- a x + b y (complex scalars, orbital blocks)."""
        self._check(x), self._check(y)
        a, b = complex(a), complex(b)
        call("inqb_axpby", self._h, x.shape[1], a.real, a.imag, x.data_ptr(), x.stride(0), b.real, b.imag,
             y.data_ptr(), y.stride(0), self._stream())
        return y

    def position_scale(self, psi, occ, direction=0, scale=1.0, out=None):
        """out = scale * occ[m] * r_dir(p) * psi (the dipole's derivative for scale = dV)."""
        psi = self._check(psi)
        out = torch.empty_like(psi) if out is None else self._check(out)
        occ_t = torch.as_tensor(occ, dtype=torch.float64, device=self.device).contiguous()
        call("inqb_position_scale", self._h, psi.data_ptr(), psi.stride(0), out.data_ptr(), out.stride(0),
             psi.shape[1], int(direction), occ_t.data_ptr(), float(scale), self._stream())
        return out

    def accum_potential_gradient_(self, gV, u, w, c=1.0):
        """gV[p] += Re(c sum_m conj(u) w) -- <u| dH/dV(p) |w>."""
        self._check(u), self._check(w)
        c = complex(c)
        call("inqb_accum_potential_gradient", self._h, u.data_ptr(), w.data_ptr(), u.shape[1], u.stride(0), c.real,
             c.imag, gV.data_ptr(), self._stream())
        return gV

    def accum_vector_potential_gradient_(self, gA, u, w, c=1.0):
        """gA[d] += Re(c <u| dH/dA_d |w>) at the current k + A (gA: 3 FP64 on the device)."""
        self._check(u), self._check(w)
        c = complex(c)
        call("inqb_accum_vector_potential_gradient", self._h, u.data_ptr(), w.data_ptr(), u.shape[1], u.stride(0),
             c.real, c.imag, gA.data_ptr(), self._stream())
        return gA

    def timing_start(self, max_applies: int):
        """Record CUDA events around the three passes of the next max_applies H applies."""
        call("inqb_timing_start", self._h, int(max_applies))

    def timing_stop(self):
        """(summed ms of [projection + tile_fwd, tile_x, tile_inv], number of timed applies)."""
        ms = np.zeros(3)
        n = ctypes.c_int(0)
        call("inqb_timing_stop", self._h, dptr(ms), ctypes.byref(n))
        return ms, n.value

    def timing_passes(self):
        """(summed ms of [projection kernel, tile_fwd, tile_x, tile_inv], number of timed applies)."""
        ms = np.zeros(4)
        n = ctypes.c_int(0)
        call("inqb_timing_passes", self._h, dptr(ms), ctypes.byref(n))
        return ms, n.value

    PROJECTION_FUSED = 0
    PROJECTION_KERNEL = 1

    def set_projection_mode(self, mode):
        """INQB_PROJECTION_FUSED (0, "fused": inside the first tile pass, the default)
        or INQB_PROJECTION_KERNEL (1, "kernel": its own gather-and-contract kernel, on
        the tensor cores in the mixed precision)."""
        self.state_version += 1
        m = {"fused": 0, "kernel": 1}.get(mode, mode)
        call("inqb_set_projection_mode", self._h, int(m))

    def device_status(self):
        """Raise if a kernel's bounded device-side wait gave up since the last check."""
        call("inqb_device_status", self._h, self._stream())

    def band_energies(self, psi, hpsi=None) -> np.ndarray:
        """eps[m] = Re<H psi_m|psi_m> / <psi_m|psi_m> (FP64 sums); H psi is applied
        here when not given."""
        psi = self._check(psi)
        if hpsi is None:
            hpsi = self.apply(psi)
        hpsi = self._check(hpsi)
        if hpsi.shape != psi.shape or hpsi.stride(0) != psi.stride(0):
            raise ValueError("psi and hpsi must have the same shape and leading dimension")
        eps = np.zeros(psi.shape[1])
        call("inqb_band_energies", self._h, psi.data_ptr(), hpsi.data_ptr(), psi.shape[1], psi.stride(0), dptr(eps),
             self._stream())
        return eps

    def orthonormalize_(self, psi):
        psi = self._check(psi)
        call("inqb_orthonormalize", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), self._stream())
        return psi

    # -- the pieces of an orbital-sharded TD-MLWF step (parallel.sharded_mlwf_step_)
    def mlwf_gram_block(self, a, b) -> torch.Tensor:
        """Z [3, Ma, Mb] complex128: sum_p conj(a_m) e^{i 2 pi r_d / |a_d|} b_n."""
        a = self._check(a)
        b = self._check(b)
        Z = torch.empty((3, a.shape[1], b.shape[1]), dtype=torch.complex128, device=a.device)
        call("inqb_mlwf_gram_block", self._h, a.data_ptr(), a.shape[1], a.stride(0), b.data_ptr(), b.shape[1],
             b.stride(0), Z.data_ptr(), self._stream())
        return Z

    def mlwf_finish(self, Z: torch.Tensor, norms: torch.Tensor) -> torch.Tensor:
        """The six [M, M] matrices of tdmlwf_trans::update from the summed Z [3, M, M]
        and the orbital norms sum_p |psi_m|^2 (FP64 [M])."""
        Z = Z.contiguous()
        norms = norms.to(torch.float64).contiguous()
        M = Z.shape[1]
        a = torch.empty((6, M, M), dtype=torch.complex128, device=Z.device)
        call("inqb_mlwf_finish", self._h, M, Z.data_ptr(), norms.data_ptr(), a.data_ptr(), self._stream())
        return a

    def orbital_norms(self, psi) -> torch.Tensor:
        """sum_p |psi_m|^2 (FP64 [M] on the device)."""
        psi = self._check(psi)
        out = torch.empty(psi.shape[1], dtype=torch.float64, device=psi.device)
        call("inqb_orbital_norms", self._h, psi.data_ptr(), psi.shape[1], psi.stride(0), out.data_ptr(),
             self._stream())
        return out

    def mlwf_centres(self, adiag):
        """(centres [M, 3], spreads [M]) from adiag [6, M] (tdmlwf_trans::center / spread2)."""
        ad = np.ascontiguousarray(torch.as_tensor(adiag).cpu().numpy(), np.complex128)
        M = ad.shape[1]
        c = np.zeros((M, 3))
        sp = np.zeros(M)
        call("inqb_mlwf_centres", self._h, M, dptr(ad.view(np.float64)), dptr(c), dptr(sp))
        return c, sp

    # -- the pieces of an orbital-sharded orthonormalisation (parallel.sharded_orthonormalize_)
    def overlap_block(self, a, b) -> torch.Tensor:
        """dV a^H b in FP64: a [N, Ma], b [N, Mb] -> complex128 [Ma, Mb] on the device
        (one block of operations::overlap's set-parallel branch)."""
        a = self._check(a)
        b = self._check(b)
        S = torch.empty((a.shape[1], b.shape[1]), dtype=torch.complex128, device=a.device)
        call("inqb_overlap_block", self._h, a.data_ptr(), a.shape[1], a.stride(0), b.data_ptr(), b.shape[1],
             b.stride(0), S.data_ptr(), S.stride(0), self._stream())
        return S

    def cholesky_inverse_(self, S: torch.Tensor) -> torch.Tensor:
        """S (complex128 [M, M] on the device, Hermitian) <- U^-1 where S = U^H U."""
        if S.dtype != torch.complex128 or not S.is_cuda or S.dim() != 2 or S.shape[0] != S.shape[1] \
                or S.stride(1) != 1:
            raise ValueError("S must be a square row-major complex128 CUDA matrix")
        call("inqb_cholesky_inverse", self._h, S.data_ptr(), S.shape[0], S.stride(0), self._stream())
        return S

    def rotate_block(self, a, R: torch.Tensor, out=None) -> torch.Tensor:
        """a R: a [N, Ma] in the context precision, R complex128 [Ma, Mo] on the device."""
        a = self._check(a)
        if R.dtype != torch.complex128 or not R.is_cuda or R.dim() != 2 or R.shape[0] != a.shape[1]:
            raise ValueError("R must be a complex128 CUDA matrix with a.shape[1] rows")
        R = R.contiguous()
        if out is None:
            out = torch.empty((a.shape[0], R.shape[1]), dtype=a.dtype, device=a.device)
        out = self._check(out)
        if R.shape[1] > 0:
            call("inqb_rotate_block", self._h, a.data_ptr(), a.shape[1], a.stride(0), R.data_ptr(), R.stride(0),
                 R.shape[1], out.data_ptr(), out.stride(0), self._stream())
        return out
