"""Python binding of the sbdx C-ABI (include/sbdx.h) over the in-tree CUDA
library libsbdx.so (sm_100a).

This is the thin layer the tests, the benchmark and the autograd check use; the
drop-in for C++ callers of the reference is the header API in
cpp/include/sbd/sbd.h. There is no CPU fallback: if the CUDA library is not
built, importing a Context raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import synth  # noqa: F401

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libsbdx.so")

SBDX_OK = 0
SBDX_FP64 = 0
SBDX_FP32 = 1
ERRORS = {1: "SBDX_ERR_ARG", 2: "SBDX_ERR_CUDA", 3: "SBDX_ERR_STATE", 4: "SBDX_ERR_NOMEM", 5: "SBDX_ERR_NUMERIC"}

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint64)

EXPORTS = [
    "sbdx_ctx_create", "sbdx_ctx_destroy", "sbdx_last_error", "sbdx_set_stream", "sbdx_launch_count",
    "sbdx_set_integrals", "sbdx_set_strings", "sbdx_build_connectivity", "sbdx_connectivity_size",
    "sbdx_get_connectivity", "sbdx_diag_terms", "sbdx_sigma", "sbdx_sigma_device", "sbdx_davidson",
    "sbdx_rdm", "sbdx_occupation", "sbdx_alpha_weights", "sbdx_energy_backward", "sbdx_set_profiling",
    "sbdx_phase_times", "sbdx_set_tuning", "sbdx_autotune", "sbdx_davidson_roots",
    "sbdx_build_hamiltonian", "sbdx_release_hamiltonian", "sbdx_wavefunction_device", "sbdx_get_wavefunction",
    "sbdx_rdm_device", "sbdx_occupation_device", "sbdx_alpha_weights_device", "sbdx_energy_backward_device",
    "sbdx_sigma_rows_device", "sbdx_set_graph_steps", "sbdx_project_device", "sbdx_set_io_chunks",
]
PHASES = ["alpha_same_spin", "transpose", "beta_same_spin", "alpha_beta", "combine"]


class DavidsonParams(ctypes.Structure):
    _fields_ = [("max_it", ctypes.c_int), ("max_nb", ctypes.c_int), ("eps", ctypes.c_double),
                ("max_time", ctypes.c_double), ("precision", ctypes.c_int), ("defect_every", ctypes.c_int),
                ("verbose", ctypes.c_int)]


class DavidsonInfo(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("residual", ctypes.c_double), ("n_sigma", ctypes.c_int),
                ("n_sigma64", ctypes.c_int), ("converged", ctypes.c_int), ("seconds", ctypes.c_double)]


class SbdxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libsbdx.so and declare the C-ABI signatures. Raises when missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"sbdx CUDA library not built: {path} (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    lib.sbdx_last_error.restype = ctypes.c_char_p
    lib.sbdx_launch_count.restype = ctypes.c_ulonglong
    lib.sbdx_ctx_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    for name in EXPORTS:
        fn = getattr(lib, name)
        if name not in ("sbdx_last_error", "sbdx_launch_count", "sbdx_phase_times"):
            fn.restype = ctypes.c_int
    lib.sbdx_phase_times.restype = ctypes.c_longlong
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _u(a):
    return a.ctypes.data_as(_up)


class Context:
    """One Hamiltonian + one alpha x beta basis on one GPU."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.sbdx_ctx_create(ctypes.byref(h), device)
        if rc != SBDX_OK:
            raise SbdxError(rc, "context creation failed (no CUDA device?)")
        self.h = h
        self.L = 0
        self.na = self.nb = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.sbdx_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != SBDX_OK:
            raise SbdxError(rc, self.lib.sbdx_last_error(self.h).decode())

    @property
    def launches(self) -> int:
        return int(self.lib.sbdx_launch_count(self.h))

    def set_profiling(self, on: bool):
        self._check(self.lib.sbdx_set_profiling(self.h, ctypes.c_int(1 if on else 0)))

    def phase_times(self):
        ms = np.zeros(len(PHASES))
        n = self.lib.sbdx_phase_times(self.h, _d(ms), ctypes.c_int(len(PHASES)))
        return int(n), dict(zip(PHASES, ms.tolist()))

    def set_tuning(self, same_vec: int = 0, ab_rows: int = 0):
        self._check(self.lib.sbdx_set_tuning(self.h, ctypes.c_int(same_vec), ctypes.c_int(ab_rows)))

    def autotune(self):
        v, r = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.sbdx_autotune(self.h, ctypes.byref(v), ctypes.byref(r)))
        return v.value, r.value

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.sbdx_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def set_integrals(self, L, I0, h, eri):
        h = np.ascontiguousarray(h, dtype=np.float64).reshape(-1)
        eri = np.ascontiguousarray(eri, dtype=np.float64)
        self._check(self.lib.sbdx_set_integrals(self.h, ctypes.c_int(L), ctypes.c_double(I0), _d(h), _d(eri),
                                                ctypes.c_size_t(len(eri))))
        self.L = L

    def set_strings(self, alpha, beta):
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        b = np.ascontiguousarray(beta, dtype=np.uint64)
        self._check(self.lib.sbdx_set_strings(self.h, _u(a), ctypes.c_size_t(len(a)), _u(b), ctypes.c_size_t(len(b))))
        self.na, self.nb = len(a), len(b)

    def load(self, prob):
        self.set_integrals(prob.L, prob.I0, prob.h, prob.eri)
        self.set_strings(prob.alpha, prob.beta)
        return self

    def build_connectivity(self):
        self._check(self.lib.sbdx_build_connectivity(self.h))

    def build_hamiltonian(self) -> int:
        """Stores H on the device (the reference's method 1); FP64 sigmas then
        use it. Returns the number of stored off-diagonal elements."""
        n = ctypes.c_uint64(0)
        self._check(self.lib.sbdx_build_hamiltonian(self.h, ctypes.byref(n)))
        return int(n.value)

    def release_hamiltonian(self):
        self._check(self.lib.sbdx_release_hamiltonian(self.h))

    def connectivity(self, spin):
        n = ctypes.c_uint64(0)
        self._check(self.lib.sbdx_connectivity_size(self.h, ctypes.c_int(spin), ctypes.byref(n)))
        rows = self.na if spin == 0 else self.nb
        sl = np.zeros(rows, np.uint64)
        dl = np.zeros(rows, np.uint64)
        idx = np.zeros(max(n.value, 1), np.uint64)
        self._check(self.lib.sbdx_get_connectivity(self.h, ctypes.c_int(spin), _u(sl), _u(dl), _u(idx)))
        return sl, dl, idx[: n.value]

    def diag_terms(self):
        out = np.zeros(self.na * self.nb)
        self._check(self.lib.sbdx_diag_terms(self.h, _d(out)))
        return out

    def sigma(self, C):
        C = np.ascontiguousarray(C, dtype=np.float64)
        S = np.empty_like(C)
        self._check(self.lib.sbdx_sigma(self.h, _d(C), _d(S)))
        return S

    def sigma_host_ptr(self, c_ptr: int, s_ptr: int):
        """sbdx_sigma on raw host pointers (e.g. pinned torch tensors)."""
        self._check(self.lib.sbdx_sigma(self.h, ctypes.cast(ctypes.c_void_p(c_ptr), _dp),
                                        ctypes.cast(ctypes.c_void_p(s_ptr), _dp)))

    def sigma_device(self, precision, c_ptr: int, s_ptr: int):
        self._check(self.lib.sbdx_sigma_device(self.h, ctypes.c_int(precision), ctypes.c_void_p(c_ptr),
                                               ctypes.c_void_p(s_ptr)))

    def set_io_chunks(self, chunks: int = 0):
        """sbdx_set_io_chunks: chunks of the host-buffer sigma's copy/compute
        pipeline (0 automatic, 1 none, K >= 2 fixed)."""
        self._check(self.lib.sbdx_set_io_chunks(self.h, ctypes.c_int(chunks)))

    def set_graph_steps(self, on: bool = True):
        """sbdx_set_graph_steps: several-root solves run one CUDA graph per iteration."""
        self._check(self.lib.sbdx_set_graph_steps(self.h, ctypes.c_int(1 if on else 0)))

    def sigma_rows_device(self, precision, c_ptr: int, s_ptr: int, a0: int, a1: int):
        """Rows [a0, a1) of S = H C (sbdx_sigma_rows_device): c_ptr the whole
        input, s_ptr the (a1 - a0) * nb output rows."""
        self._check(self.lib.sbdx_sigma_rows_device(self.h, ctypes.c_int(precision), ctypes.c_void_p(c_ptr),
                                                    ctypes.c_void_p(s_ptr), ctypes.c_size_t(a0), ctypes.c_size_t(a1)))

    def project_device(self, precision, v_ptr: int, ldv: int, m: int, x_ptr: int, ldx: int, nx: int, D: int,
                       p_ptr: int):
        """sbdx_project_device: p[i * nx + r] = <V_i, X_r> on the device."""
        self._check(self.lib.sbdx_project_device(self.h, ctypes.c_int(precision), ctypes.c_void_p(v_ptr),
                                                 ctypes.c_size_t(ldv), ctypes.c_int(m), ctypes.c_void_p(x_ptr),
                                                 ctypes.c_size_t(ldx), ctypes.c_int(nx), ctypes.c_size_t(D),
                                                 ctypes.c_void_p(p_ptr)))

    def davidson(self, max_it=1, max_nb=10, eps=1e-4, max_time=86400.0, precision=SBDX_FP64, defect_every=0,
                 verbose=0, W=None, to_host=True):
        """sbdx_davidson. Returns (info, W); with to_host=False (and no start
        vector) W is None and the result stays on the device only
        (wavefunction_device)."""
        p = DavidsonParams(max_it, max_nb, eps, max_time, precision, defect_every, verbose)
        D = self.na * self.nb
        init = 1 if W is not None else 0
        if W is not None:
            W = np.ascontiguousarray(W, dtype=np.float64).copy()
        elif to_host:
            W = np.zeros(D)
        info = DavidsonInfo()
        self._check(self.lib.sbdx_davidson(self.h, ctypes.byref(p), ctypes.c_int(init), _d(W) if W is not None else None,
                                           ctypes.byref(info)))
        return info, W

    def davidson_roots(self, nroots, max_it=1, max_nb=10, eps=1e-4, max_time=86400.0, precision=SBDX_FP64,
                       defect_every=0, verbose=0, W=None, to_host=True):
        """sbdx_davidson_roots: the nroots lowest eigenpairs. Returns
        (info, energies[nroots], residuals[nroots], W[nroots, D])."""
        p = DavidsonParams(max_it, max_nb, eps, max_time, precision, defect_every, verbose)
        D = self.na * self.nb
        init = 1 if W is not None else 0
        if W is not None:
            Wb = np.ascontiguousarray(W, dtype=np.float64).reshape(nroots, D).copy()
        else:
            Wb = np.zeros((nroots, D)) if to_host else None
        E = np.zeros(nroots)
        res = np.zeros(nroots)
        info = DavidsonInfo()
        self._check(self.lib.sbdx_davidson_roots(self.h, ctypes.byref(p), ctypes.c_int(nroots), ctypes.c_int(init),
                                                 _d(Wb) if Wb is not None else None, _d(E), _d(res),
                                                 ctypes.byref(info)))
        return info, E, res, Wb

    # ---- the resident result of the last solve and reductions on device vectors ----
    def wavefunction_device(self, root=0) -> int:
        """Device address of root `root` of the last solve (sbdx_wavefunction_device)."""
        ptr = ctypes.c_void_p()
        self._check(self.lib.sbdx_wavefunction_device(self.h, ctypes.c_int(root), ctypes.byref(ptr)))
        return int(ptr.value)

    def get_wavefunction(self, root=0):
        W = np.zeros(self.na * self.nb)
        self._check(self.lib.sbdx_get_wavefunction(self.h, ctypes.c_int(root), _d(W)))
        return W

    def rdm_device(self, w_ptr: int, two=True):
        L = self.L
        one = np.zeros(2 * L * L)
        tw = np.zeros(4 * L ** 4) if two else None
        self._check(self.lib.sbdx_rdm_device(self.h, ctypes.c_void_p(w_ptr), _d(one), _d(tw) if two else None))
        return one, tw

    def occupation_device(self, w_ptr: int):
        out = np.zeros(2 * self.L)
        self._check(self.lib.sbdx_occupation_device(self.h, ctypes.c_void_p(w_ptr), _d(out)))
        return out

    def alpha_weights_device(self, w_ptr: int):
        out = np.zeros(self.na)
        self._check(self.lib.sbdx_alpha_weights_device(self.h, ctypes.c_void_p(w_ptr), _d(out)))
        return out

    def energy_backward_device(self, w_ptr: int):
        L = self.L
        dh = np.zeros(L * L)
        deri = np.zeros(synth.neri(L))
        self._check(self.lib.sbdx_energy_backward_device(self.h, ctypes.c_void_p(w_ptr), _d(dh), _d(deri)))
        return dh, deri

    def rdm(self, W, two=True):
        L = self.L
        one = np.zeros(2 * L * L)
        tw = np.zeros(4 * L ** 4) if two else None
        W = np.ascontiguousarray(W, dtype=np.float64)
        self._check(self.lib.sbdx_rdm(self.h, _d(W), _d(one), _d(tw) if two else None))
        return one, tw

    def occupation(self, W):
        out = np.zeros(2 * self.L)
        self._check(self.lib.sbdx_occupation(self.h, _d(np.ascontiguousarray(W, dtype=np.float64)), _d(out)))
        return out

    def alpha_weights(self, W):
        out = np.zeros(self.na)
        self._check(self.lib.sbdx_alpha_weights(self.h, _d(np.ascontiguousarray(W, dtype=np.float64)), _d(out)))
        return out

    def energy_backward(self, W):
        L = self.L
        dh = np.zeros(L * L)
        deri = np.zeros(synth.neri(L))
        self._check(self.lib.sbdx_energy_backward(self.h, _d(np.ascontiguousarray(W, dtype=np.float64)), _d(dh), _d(deri)))
        return dh, deri


def diag_terms_noalloc(norb: int, I0: float, h_ptr: int, eri_ptr: int, alpha_ptr: int, na: int, beta_ptr: int,
                       nb: int, hii_ptr: int, stream_ptr: int = 0):
    """sbdx_diag_terms_noalloc on caller-owned device pointers (no context, no
    device allocation). Launches asynchronously on `stream_ptr`; the library
    keeps one fixed 4 MiB scratch array per GPU, so calls must not overlap.
    Raises SbdxError with the library's message on a non-zero status."""
    lib = load_library()
    fn = lib.sbdx_diag_terms_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_char_p, ctypes.c_size_t]
    buf = ctypes.create_string_buffer(256)
    rc = fn(norb, I0, h_ptr, eri_ptr, alpha_ptr, na, beta_ptr, nb, hii_ptr, stream_ptr, buf, len(buf))
    if rc != SBDX_OK:
        raise SbdxError(rc, buf.value.decode())


class Batch:
    """sbdx_batch: many alpha x beta subspaces sharing one Hamiltonian, solved
    concurrently on one GPU (per-subspace streams, graph-replayed sigmas)."""

    def __init__(self, L, I0, h, eri, device: int = 0):
        self.lib = load_library()
        lib = self.lib
        lib.sbdx_batch_last_error.restype = ctypes.c_char_p
        lib.sbdx_batch_last_error.argtypes = [ctypes.c_void_p]
        for name in ("sbdx_batch_create", "sbdx_batch_destroy", "sbdx_batch_add", "sbdx_batch_size",
                     "sbdx_batch_dims", "sbdx_batch_tune", "sbdx_batch_solve", "sbdx_batch_vector",
                     "sbdx_batch_set_graph_steps"):
            getattr(lib, name).restype = ctypes.c_int
        h = np.ascontiguousarray(h, dtype=np.float64)
        eri = np.ascontiguousarray(eri, dtype=np.float64)
        b = ctypes.c_void_p()
        rc = lib.sbdx_batch_create(ctypes.byref(b), ctypes.c_int(device), ctypes.c_int(L), ctypes.c_double(I0), _d(h),
                                   _d(eri), ctypes.c_size_t(len(eri)))
        if rc != SBDX_OK:
            raise SbdxError(rc, "batch creation failed")
        self.b = b
        self.dims = []

    def _check(self, rc):
        if rc != SBDX_OK:
            raise SbdxError(rc, self.lib.sbdx_batch_last_error(self.b).decode())

    def close(self):
        if getattr(self, "b", None):
            self.lib.sbdx_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, alpha, beta) -> int:
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        b = np.ascontiguousarray(beta, dtype=np.uint64)
        idx = ctypes.c_int(-1)
        self._check(self.lib.sbdx_batch_add(self.b, _u(a), ctypes.c_size_t(len(a)), _u(b), ctypes.c_size_t(len(b)),
                                            ctypes.byref(idx)))
        self.dims.append((len(a), len(b)))
        return idx.value

    def set_graph_steps(self, on: bool = True):
        self._check(self.lib.sbdx_batch_set_graph_steps(self.b, ctypes.c_int(1 if on else 0)))

    def tune(self):
        s, a = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.sbdx_batch_tune(self.b, ctypes.byref(s), ctypes.byref(a)))
        return s.value, a.value

    def solve(self, nroots=1, max_it=100, max_nb=12, eps=1e-8, precision=SBDX_FP64, nthreads=0, max_time=86400.0,
              defect_every=0):
        """Returns (energies[K, nroots], residuals[K, nroots], infos[K], seconds)."""
        K = len(self.dims)
        p = DavidsonParams(max_it, max_nb, eps, max_time, precision, defect_every, 0)
        E = np.zeros((K, nroots))
        R = np.zeros((K, nroots))
        infos = (DavidsonInfo * K)()
        sec = ctypes.c_double(0.0)
        self._check(self.lib.sbdx_batch_solve(self.b, ctypes.byref(p), ctypes.c_int(nroots), ctypes.c_int(nthreads),
                                              _d(E), _d(R), infos, ctypes.byref(sec)))
        return E, R, list(infos), sec.value

    def vector(self, index, root=0):
        na, nb = self.dims[index]
        W = np.zeros(na * nb)
        self._check(self.lib.sbdx_batch_vector(self.b, ctypes.c_int(index), ctypes.c_int(root), _d(W)))
        return W
