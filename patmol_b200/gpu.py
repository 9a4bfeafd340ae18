"""Python host mirror of the reference's integral / Fock-build interface over
the C ABI of libpatgpu.so (include/patgpu.h).

The class ``GpuBasis`` plays the role of the reference's basis module plus
ERIFS handle: ``two_electron_ints`` builds the screened quartet list,
``rhf_form_gmatrix`` / ``uhf_form_gmatrix`` accumulate G into packed lower
triangles exactly like scfaux.c:429-714, ``dpm_ints`` subtracts the DPM
potential (dpmints.c:121-199) and ``one_electron_ints`` fills S, T, H
(oneints.c:139-234).  Failures raise ``PatgpuError``; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpatgpu.so")

_lib = None


class PatgpuError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    """Compile libpatgpu.so for sm_100a (nvcc; no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", f"-j{max(1, os.cpu_count() or 1)}", "-C", os.path.join(HERE, "csrc")],
                       check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PatgpuError(f"{LIB_PATH} is missing: build it with `make -C patmol_b200/csrc`")
        L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lp = ctypes.POINTER(ctypes.c_longlong)
        H = ctypes.c_void_p
        L.patgpu_last_error.restype = ctypes.c_int
        L.patgpu_error_message.restype = ctypes.c_char_p
        L.patgpu_basis_create.argtypes = [ctypes.c_int, ip, ip, ip, ip, ip, dp, dp, ctypes.c_int, dp, dp,
                                          ctypes.c_int, ctypes.c_double, ctypes.POINTER(H)]
        L.patgpu_basis_destroy.argtypes = [H]
        L.patgpu_set_quartets.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.patgpu_rhf_gmatrix.argtypes = [H, dp, dp]
        L.patgpu_uhf_gmatrix.argtypes = [H, dp, dp, dp, dp]
        L.patgpu_jk.argtypes = [H, dp, dp, dp]
        L.patgpu_rhf_gmatrix_device.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.patgpu_rhf_accumulate_device.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.patgpu_finish_gmatrix_device.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.patgpu_rhf_gmatrix_device_noalloc.argtypes = [H, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.patgpu_eri_quartets.argtypes = [H, ctypes.c_int, ip, dp]
        L.patgpu_oneints.argtypes = [H, dp, dp, dp]
        L.patgpu_dpm.argtypes = [H, dp]
        L.patgpu_onebody.argtypes = [ctypes.c_int, ip, ip, ip, ip, ip, dp, dp, ctypes.c_int, dp, dp, ctypes.c_int,
                                     dp, dp, dp, dp]
        L.patgpu_stats.argtypes = [H, lp]
        L.patgpu_class_counts.argtypes = [H, ctypes.c_int, ip, lp]
        L.patgpu_last_timing.argtypes = [H, dp, ip]
        L.patgpu_rys_host.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.patgpu_fp64_peak.argtypes = [dp]
        L.patgpu_dmma_peak.argtypes = [dp]
        L.patgpu_set_mixed_precision.argtypes = [H, ctypes.c_double]
        L.patgpu_set_deterministic.argtypes = [H, ctypes.c_int]
        L.patgpu_moments.argtypes = [ctypes.c_int, ip, ip, ip, ip, ip, dp, dp, ctypes.c_int, dp, dp, dp]
        L.patgpu_accumulator_bytes.argtypes = [H, ctypes.POINTER(ctypes.c_size_t)]
        L.patgpu_mixed_stats.argtypes = [H, lp]
        L.patgpu_rhf_gradient.argtypes = [H, dp, dp, ctypes.c_int, ctypes.c_int, dp]
        L.patgpu_uhf_gradient.argtypes = [H, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, dp]
        L.patgpu_write_eri_files.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                             ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, ip, ip]
        L.patgpu_scf_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ctypes.POINTER(H)]
        L.patgpu_scf_destroy.argtypes = [H]
        L.patgpu_scf_density_host.argtypes = [H, dp, dp, dp, dp, dp]
        L.patgpu_set_density_screening.argtypes = [H, ctypes.c_double]
        L.patgpu_set_density_precision.argtypes = [H, ctypes.c_double]
        L.patgpu_batch_set_density_screening.argtypes = [H, ctypes.c_double, ctypes.c_double]
        L.patgpu_batch_set_density_thresholds.argtypes = [H, dp, dp]
        L.patgpu_batch_last_computed.argtypes = [H, lp]
        L.patgpu_last_computed.argtypes = [H, lp]
        L.patgpu_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(H), ctypes.POINTER(H)]
        L.patgpu_batch_destroy.argtypes = [H]
        L.patgpu_batch_buffers.argtypes = [H, ctypes.c_int, ctypes.POINTER(dp), ctypes.POINTER(dp)]
        L.patgpu_batch_set_mixed_precision.argtypes = [H, ctypes.c_double]
        L.patgpu_batch_launch.argtypes = [H, ctypes.c_void_p]
        L.patgpu_batch_rhf_gmatrix.argtypes = [H, ctypes.POINTER(dp), ctypes.POINTER(dp)]
        L.patgpu_batch_stats.argtypes = [H, lp]
        L.patgpu_batch_last_timing.argtypes = [H, dp]
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _check(rc: int, what: str):
    if rc != 0:
        msg = lib().patgpu_error_message().decode(errors="replace")
        raise PatgpuError(f"{what}: {msg} (code {rc})")


def fp64_peak_tflops() -> float:
    v = ctypes.c_double()
    _check(lib().patgpu_fp64_peak(ctypes.byref(v)), "patgpu_fp64_peak")
    return v.value


def dmma_peak_tflops() -> float:
    """FP64 mma.sync (DMMA) rate of this GPU, TFLOP/s."""
    t = ctypes.c_double()
    _check(lib().patgpu_dmma_peak(ctypes.byref(t)), "patgpu_dmma_peak")
    return t.value


def rys_host(n: int, T: float):
    """Nodes (t^2) and weights of the tables the kernels use, evaluated on the host."""
    x = np.zeros(n)
    w = np.zeros(n)
    _check(lib().patgpu_rys_host(n, float(T), _p(x), _p(w)), "patgpu_rys_host")
    return x, w


class GpuBasis:
    """A basis bound to the current CUDA device (see patgpu_basis_create)."""

    def __init__(self, basis, schwarz_tau: float = 1e-14):
        self.basis = basis
        self.n = basis.norb
        self.no2 = self.n * (self.n + 1) // 2
        self._f = basis.flat_arrays()
        f = self._f
        h = ctypes.c_void_p()
        _check(lib().patgpu_basis_create(basis.nshell, _p(f["l"], ctypes.c_int), _p(f["cen"], ctypes.c_int),
                                         _p(f["off"], ctypes.c_int), _p(f["nst"], ctypes.c_int),
                                         _p(f["prim_off"], ctypes.c_int), _p(f["alpha"]), _p(f["coef"]),
                                         basis.ncen, _p(f["charges"]), _p(f["coords"]), basis.skipcen,
                                         float(schwarz_tau), ctypes.byref(h)), "patgpu_basis_create")
        self.h = h

    def close(self):
        if self.h:
            lib().patgpu_basis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference-shaped interface -------------------------------------
    def two_electron_ints(self, start: int = 0, rank: int = 0, nranks: int = 1):
        _check(lib().patgpu_set_quartets(self.h, start, rank, nranks), "two_electron_ints")

    def rhf_form_gmatrix(self, P, G=None):
        P = np.ascontiguousarray(P, dtype=np.float64)
        G = np.zeros(self.no2) if G is None else G
        _check(lib().patgpu_rhf_gmatrix(self.h, _p(P), _p(G)), "rhf_form_gmatrix")
        return G

    def uhf_form_gmatrix(self, PA, PB, GA=None, GB=None):
        PA = np.ascontiguousarray(PA, dtype=np.float64)
        PB = np.ascontiguousarray(PB, dtype=np.float64)
        GA = np.zeros(self.no2) if GA is None else GA
        GB = np.zeros(self.no2) if GB is None else GB
        _check(lib().patgpu_uhf_gmatrix(self.h, _p(PA), _p(PB), _p(GA), _p(GB)), "uhf_form_gmatrix")
        return GA, GB

    def jk(self, P):
        P = np.ascontiguousarray(P, dtype=np.float64)
        J = np.zeros(self.no2)
        K = np.zeros(self.no2)
        _check(lib().patgpu_jk(self.h, _p(P), _p(J), _p(K)), "patgpu_jk")
        return J, K

    def one_electron_ints(self):
        S, T, H = np.zeros(self.no2), np.zeros(self.no2), np.zeros(self.no2)
        _check(lib().patgpu_oneints(self.h, _p(S), _p(T), _p(H)), "one_electron_ints")
        return S, T, H

    def dpm_ints(self, H):
        H = np.array(H, dtype=np.float64)
        _check(lib().patgpu_dpm(self.h, _p(H)), "dpm_ints")
        return H

    # -- extras -----------------------------------------------------------
    def eri_quartets(self, quartets):
        q = np.ascontiguousarray(np.asarray(quartets, dtype=np.int32).reshape(-1, 4))
        sh = self.basis.shells
        sizes = [sh[a].nst * sh[b].nst * sh[c].nst * sh[d].nst for a, b, c, d in q]
        out = np.zeros(int(sum(sizes)))
        _check(lib().patgpu_eri_quartets(self.h, len(q), _p(q, ctypes.c_int), _p(out)), "patgpu_eri_quartets")
        blocks, o = [], 0
        for (a, b, c, d), s in zip(q, sizes):
            blocks.append(out[o:o + s].reshape(sh[a].nst, sh[b].nst, sh[c].nst, sh[d].nst))
            o += s
        return blocks

    def rhf_gmatrix_device(self, dP_ptr: int, dG_ptr: int, stream: int):
        """stream: the raw cudaStream_t handle (e.g. torch.cuda.Stream.cuda_stream)."""
        _check(lib().patgpu_rhf_gmatrix_device(self.h, dP_ptr, dG_ptr, stream), "rhf_gmatrix_device")

    def rhf_gmatrix_device_noalloc(self, dP_ptr: int, dG_ptr: int, stream: int):
        """Same result as rhf_gmatrix_device without any device allocation
        (working matrices in the library's fixed scratch; n <= 512)."""
        _check(lib().patgpu_rhf_gmatrix_device_noalloc(self.h, dP_ptr, dG_ptr, stream),
               "rhf_gmatrix_device_noalloc")

    def rhf_accumulate_device(self, dP_ptr: int, dA_ptr: int, stream: int):
        _check(lib().patgpu_rhf_accumulate_device(self.h, dP_ptr, dA_ptr, stream), "accumulate")

    def set_deterministic(self, on: bool):
        """Exact fixed-point J/K accumulation (bitwise reproducible G; the
        default) or FP64 atomic adds."""
        _check(lib().patgpu_set_deterministic(self.h, 1 if on else 0), "set_deterministic")

    def accumulator_bytes(self) -> int:
        """Size of the accumulator rhf_accumulate_device fills (16 n^2 bytes
        with deterministic accumulation, 8 n^2 without)."""
        b = ctypes.c_size_t(0)
        _check(lib().patgpu_accumulator_bytes(self.h, ctypes.byref(b)), "accumulator_bytes")
        return int(b.value)

    def finish_gmatrix_device(self, dA_ptr: int, dG_ptr: int, stream: int):
        _check(lib().patgpu_finish_gmatrix_device(self.h, dA_ptr, dG_ptr, stream), "finish")

    GRAD_2E, GRAD_1E, GRAD_NUC, GRAD_ALL = 1, 2, 4, 7

    def rhf_gradient(self, P, W=None, parts: int = 7, with_dpm: bool = False):
        """Nuclear gradient (ncen x 3) of E = 2 tr(PH) + tr(P G[P]) + E_nuc at
        the packed half density P and energy-weighted density W; parts is a
        mask of GRAD_2E / GRAD_1E / GRAD_NUC (patgpu_rhf_gradient)."""
        P = np.ascontiguousarray(P, dtype=np.float64)
        null = ctypes.POINTER(ctypes.c_double)()
        Wp = null
        if W is not None:
            W = np.ascontiguousarray(W, dtype=np.float64)
            Wp = _p(W)
        g = np.zeros(3 * self.basis.ncen)
        _check(lib().patgpu_rhf_gradient(self.h, _p(P), Wp, int(parts), int(bool(with_dpm)), _p(g)),
               "patgpu_rhf_gradient")
        return g.reshape(-1, 3)

    def uhf_gradient(self, PA, PB, WA=None, WB=None, parts: int = 7, with_dpm: bool = False):
        """Nuclear gradient (ncen x 3) of the UHF energy at the packed spin
        densities and energy-weighted spin densities (patgpu_uhf_gradient)."""
        arrs = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None for x in (PA, PB, WA, WB)]
        null = ctypes.POINTER(ctypes.c_double)()
        ptr = [(_p(x) if x is not None else null) for x in arrs]
        g = np.zeros(3 * self.basis.ncen)
        _check(lib().patgpu_uhf_gradient(self.h, ptr[0], ptr[1], ptr[2], ptr[3], int(parts), int(bool(with_dpm)),
                                         _p(g)), "patgpu_uhf_gradient")
        return g.reshape(-1, 3)

    def write_eri_files(self, prefix: str, basename: str, start: int = 0, rank: int = 0, nproc: int = 1,
                        max_records: int = (1 << 30) // 16, max_files: int = 4096):
        """Write the reference's ERI files (patgpu_write_eri_files); returns the
        record count of each file, named prefix + rank + file number + basename."""
        numints = np.zeros(max_files, dtype=np.int32)
        nf = ctypes.c_int()
        _check(lib().patgpu_write_eri_files(self.h, start, rank, nproc, prefix.encode(), basename.encode(),
                                            int(max_records), max_files, _p(numints, ctypes.c_int),
                                            ctypes.byref(nf)), "patgpu_write_eri_files")
        return [int(x) for x in numints[:nf.value]]

    def set_density_screening(self, tau_dens: float):
        """Skip quartets with Q_ab Q_cd max|D| < tau_dens in host-buffer builds
        (for incremental builds over density differences); 0 turns it off."""
        _check(lib().patgpu_set_density_screening(self.h, float(tau_dens)), "set_density_screening")

    def last_computed(self) -> int:
        n = ctypes.c_longlong()
        _check(lib().patgpu_last_computed(self.h, ctypes.byref(n)), "patgpu_last_computed")
        return n.value

    def set_density_precision(self, tau32: float):
        """In density-screened builds, FP32 arithmetic (FP64 sums) for kept
        quartets whose bound Q_ab Q_cd max|D| is below tau32; 0 turns it off."""
        _check(lib().patgpu_set_density_precision(self.h, float(tau32)), "set_density_precision")

    def set_mixed_precision(self, tau_fp32: float) -> int:
        """FP32 arithmetic for quartets whose Rys-term bound is below
        tau_fp32 (FP64 accumulation); returns how many quartets run in FP32."""
        _check(lib().patgpu_set_mixed_precision(self.h, float(tau_fp32)), "set_mixed_precision")
        n = ctypes.c_longlong()
        _check(lib().patgpu_mixed_stats(self.h, ctypes.byref(n)), "mixed_stats")
        return n.value

    def stats(self):
        o = np.zeros(5, dtype=np.int64)
        _check(lib().patgpu_stats(self.h, _p(o, ctypes.c_longlong)), "patgpu_stats")
        return dict(n=int(o[0]), pairs=int(o[1]), quartets=int(o[2]), classes=int(o[3]), unscreened=int(o[4]))

    def class_counts(self):
        l4 = np.zeros(4 * 128, dtype=np.int32)
        c = np.zeros(128, dtype=np.int64)
        k = lib().patgpu_class_counts(self.h, 128, _p(l4, ctypes.c_int), _p(c, ctypes.c_longlong))
        return [(tuple(int(v) for v in l4[4 * i:4 * i + 4]), int(c[i])) for i in range(k)]

    def last_timing(self):
        ns = ctypes.c_double()
        n = ctypes.c_int()
        _check(lib().patgpu_last_timing(self.h, ctypes.byref(ns), ctypes.byref(n)), "patgpu_last_timing")
        return ns.value, n.value


class GpuBatch:
    """Lock-step Fock builds of many molecules as one CUDA graph
    (patgpu_batch_*).  The GpuBasis objects must outlive the batch."""

    def __init__(self, gpu_bases):
        self.mols = list(gpu_bases)
        arr = (ctypes.c_void_p * len(self.mols))(*[g.h for g in self.mols])
        b = ctypes.c_void_p()
        _check(lib().patgpu_batch_create(len(self.mols), arr, ctypes.byref(b)), "patgpu_batch_create")
        self.b = b

    def close(self):
        if self.b:
            lib().patgpu_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_mixed_precision(self, tau_fp32: float):
        _check(lib().patgpu_batch_set_mixed_precision(self.b, float(tau_fp32)), "batch mixed precision")

    def set_density_screening(self, tau_dens: float, tau32: float = 0.0):
        """Density screening (and density-weighted FP32, tau32) of every
        molecule's build: launches then replay the screened graph."""
        _check(lib().patgpu_batch_set_density_screening(self.b, float(tau_dens), float(tau32)),
               "batch_set_density_screening")

    def set_density_thresholds(self, tau_dens, tau32=None):
        """Per-molecule density screening thresholds (and density-weighted
        FP32 thresholds); the screened graph reads them at every launch."""
        t = np.ascontiguousarray(tau_dens, dtype=np.float64)
        t32 = np.zeros_like(t) if tau32 is None else np.ascontiguousarray(tau32, dtype=np.float64)
        if t.shape != (len(self.mols),) or t32.shape != t.shape:
            raise ValueError("one threshold per molecule")
        _check(lib().patgpu_batch_set_density_thresholds(self.b, _p(t, ctypes.c_double), _p(t32, ctypes.c_double)),
               "batch_set_density_thresholds")

    def last_computed(self) -> int:
        n = ctypes.c_longlong()
        _check(lib().patgpu_batch_last_computed(self.b, ctypes.byref(n)), "batch_last_computed")
        return n.value

    def rhf_form_gmatrix(self, Ps):
        """G_m = G[P_m] for every molecule (packed host arrays)."""
        Ps = [np.ascontiguousarray(P, dtype=np.float64) for P in Ps]
        Gs = [np.zeros(g.no2) for g in self.mols]
        dp = ctypes.POINTER(ctypes.c_double)
        pa = (dp * len(Ps))(*[_p(P) for P in Ps])
        ga = (dp * len(Gs))(*[_p(G) for G in Gs])
        _check(lib().patgpu_batch_rhf_gmatrix(self.b, pa, ga), "patgpu_batch_rhf_gmatrix")
        return Gs

    def buffers(self, m: int):
        """Device addresses of molecule m's packed P and G buffers."""
        dP = ctypes.POINTER(ctypes.c_double)()
        dG = ctypes.POINTER(ctypes.c_double)()
        _check(lib().patgpu_batch_buffers(self.b, m, ctypes.byref(dP), ctypes.byref(dG)), "batch buffers")
        return ctypes.cast(dP, ctypes.c_void_p).value, ctypes.cast(dG, ctypes.c_void_p).value

    def launch(self, stream: int):
        _check(lib().patgpu_batch_launch(self.b, stream), "patgpu_batch_launch")

    def stats(self):
        o = np.zeros(4, dtype=np.int64)
        _check(lib().patgpu_batch_stats(self.b, _p(o, ctypes.c_longlong)), "patgpu_batch_stats")
        return dict(molecules=int(o[0]), quartets=int(o[1]), fp32_quartets=int(o[2]), graph_nodes=int(o[3]))

    def last_timing_ns(self) -> float:
        v = ctypes.c_double()
        _check(lib().patgpu_batch_last_timing(self.b, ctypes.byref(v)), "patgpu_batch_last_timing")
        return v.value


class GpuScfLinalg:
    """SCF linear algebra on the GPU (patgpu_scf_*): from a Fock matrix, the
    orbitals, the half density P and the energy-weighted density W."""

    def __init__(self, X, nocc: int):
        X = np.ascontiguousarray(X, dtype=np.float64)
        self.n, self.nx = X.shape
        self.nocc = nocc
        s = ctypes.c_void_p()
        _check(lib().patgpu_scf_create(self.n, self.nx, nocc, _p(X), ctypes.byref(s)), "patgpu_scf_create")
        self.s = s

    def close(self):
        if self.s:
            lib().patgpu_scf_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def density(self, F_packed):
        """Returns (eps, C (n x nx), P packed, W packed)."""
        F = np.ascontiguousarray(F_packed, dtype=np.float64)
        no2 = self.n * (self.n + 1) // 2
        P, W = np.empty(no2), np.empty(no2)
        eps = np.empty(self.nx)
        Ccm = np.empty((self.nx, self.n))
        _check(lib().patgpu_scf_density_host(self.s, _p(F), _p(P), _p(W), _p(eps), _p(Ccm)),
               "patgpu_scf_density_host")
        return eps, Ccm.T.copy(), P, W


ERINT_DTYPE = np.dtype([("val", "<f8"), ("i", "<u2"), ("j", "<u2"), ("k", "<u2"), ("l", "<u2")])


def read_eri_files(prefix: str, basename: str, rank: int, nfiles: int):
    """Concatenated records of ERI files f = 0 .. nfiles-1 (ERINT layout, erifs.h:19-22)."""
    parts = [np.fromfile(f"{prefix}{rank}{f}{basename}", dtype=ERINT_DTYPE) for f in range(nfiles)]
    return np.concatenate(parts) if parts else np.zeros(0, dtype=ERINT_DTYPE)


def moments(basis):
    """Dipole (3, no2) and quadrupole (6, no2: xx, xy, xz, yy, yz, zz)
    integrals about the origin, packed (patgpu_moments, momints.c)."""
    f = basis.flat_arrays()
    no2 = basis.norb * (basis.norb + 1) // 2
    dip = np.zeros(3 * no2)
    quad = np.zeros(6 * no2)
    _check(lib().patgpu_moments(basis.nshell, _p(f["l"], ctypes.c_int), _p(f["cen"], ctypes.c_int),
                                _p(f["off"], ctypes.c_int), _p(f["nst"], ctypes.c_int),
                                _p(f["prim_off"], ctypes.c_int), _p(f["alpha"]), _p(f["coef"]), basis.ncen,
                                _p(f["coords"]), _p(dip), _p(quad)), "patgpu_moments")
    return dip.reshape(3, no2), quad.reshape(6, no2)


def onebody(basis, want_sth=True, Hdpm=None):
    """Handle-free one-body integrals (patgpu_onebody)."""
    f = basis.flat_arrays()
    no2 = basis.norb * (basis.norb + 1) // 2
    S = T = H = None
    null = ctypes.POINTER(ctypes.c_double)()
    if want_sth:
        S, T, H = np.zeros(no2), np.zeros(no2), np.zeros(no2)
    if Hdpm is not None:
        Hdpm = np.array(Hdpm, dtype=np.float64)
    _check(lib().patgpu_onebody(basis.nshell, _p(f["l"], ctypes.c_int), _p(f["cen"], ctypes.c_int),
                                _p(f["off"], ctypes.c_int), _p(f["nst"], ctypes.c_int),
                                _p(f["prim_off"], ctypes.c_int), _p(f["alpha"]), _p(f["coef"]), basis.ncen,
                                _p(f["charges"]), _p(f["coords"]), basis.skipcen,
                                _p(S) if want_sth else null, _p(T) if want_sth else null,
                                _p(H) if want_sth else null, _p(Hdpm) if Hdpm is not None else null),
           "patgpu_onebody")
    return S, T, H, Hdpm
