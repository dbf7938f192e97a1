"""ctypes access to the CPU checkers (TEST INFRASTRUCTURE ONLY).

Two checkers live under oracle/:
  * ``Port``  -- liboracle.so, our C restatement of the reference algorithm
                 (oracle/sbd_oracle.c);
  * ``Ref``   -- oracle/_ref/libsbdref.so, the unmodified reference headers
                 (walkup/sbd-ykt include/sbd) compiled with the serial MPI shim
                 by oracle/Makefile (present where it was built).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module. Arrays follow the product conventions: one uint64 per spin string,
alpha-major vectors, L*L one-body matrix, 8-fold packed ERI.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsbdref.so")
REF_CLI = os.path.join(HERE, "_ref", "sbd_ref_cli")

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint64)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _u(a):
    return a.ctypes.data_as(_up) if a is not None else None


def build_port() -> str:
    """Compile the C restatement (make -C oracle port)."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_SO


def reference_root() -> str:
    """Root of the reference tree: $SBD_REFERENCE, else this container's mount."""
    return os.environ.get("SBD_REFERENCE", "/root/reference")


def build_ref(ref_root: str | None = None) -> str | None:
    """Compile the reference checker when the reference tree is present."""
    ref_root = ref_root or reference_root()
    if not os.path.isdir(os.path.join(ref_root, "include", "sbd")):
        return None
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    return REF_SO


class Port:
    """The C restatement (sbd_oracle.c)."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            build_port()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.sbo_connectivity.restype = ctypes.c_longlong
        L.sbo_hij.restype = ctypes.c_double
        L.sbo_hij.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _dp] + [ctypes.c_uint64] * 4
        L.sbo_parity.restype = ctypes.c_int
        L.sbo_parity.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.sbo_davidson.restype = ctypes.c_double
        L.sbo_carryover.restype = ctypes.c_longlong
        L.sbo_rdm_energy.restype = ctypes.c_double

    def connectivity(self, s):
        s = np.ascontiguousarray(s, dtype=np.uint64)
        n = len(s)
        sl = np.zeros(n, np.uint64)
        dl = np.zeros(n, np.uint64)
        tot = self.lib.sbo_connectivity(_u(s), ctypes.c_size_t(n), _u(sl), _u(dl), None)
        idx = np.zeros(max(tot, 1), np.uint64)
        self.lib.sbo_connectivity(_u(s), ctypes.c_size_t(n), _u(sl), _u(dl), _u(idx))
        return sl, dl, idx[:tot]

    def hij(self, prob, bra_a, bra_b, ket_a, ket_b):
        return self.lib.sbo_hij(prob.L, prob.I0, _d(prob.h), _d(prob.eri), int(bra_a), int(bra_b), int(ket_a), int(ket_b))

    def parity(self, alpha, beta, start, end):
        return self.lib.sbo_parity(int(alpha), int(beta), int(start), int(end))

    def diag_terms(self, prob):
        out = np.zeros(prob.na * prob.nb)
        self.lib.sbo_diag_terms(ctypes.c_int(prob.L), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri),
                                _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb), _d(out))
        return out

    def sigma(self, prob, C, hii=None):
        C = np.ascontiguousarray(C, dtype=np.float64)
        out = np.zeros_like(C)
        self.lib.sbo_sigma(ctypes.c_int(prob.L), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri),
                           _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb),
                           _d(hii), _d(C), _d(out))
        return out

    def sigma_rows(self, prob, C, row0, rows):
        """Off-diagonal part of the bra alpha rows [row0, row0 + rows) of
        sigma: rows x nb values, row-major."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        rows = min(rows, prob.na - row0)
        out = np.zeros(rows * prob.nb)
        self.lib.sbo_sigma_rows(ctypes.c_int(prob.L), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri),
                                _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb),
                                _d(C), ctypes.c_size_t(row0), ctypes.c_size_t(rows), _d(out))
        return out

    def davidson(self, prob, max_it=1, max_nb=10, eps=1e-4, W=None):
        D = prob.na * prob.nb
        if W is None:
            W = np.zeros(D)
            W[0] = 1.0
        W = np.ascontiguousarray(W, dtype=np.float64).copy()
        ns = ctypes.c_int(0)
        E = self.lib.sbo_davidson(ctypes.c_int(prob.L), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri),
                                  _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb),
                                  ctypes.c_int(max_it), ctypes.c_int(max_nb), ctypes.c_double(eps), _d(W), ctypes.byref(ns))
        return E, W, ns.value

    def rdm(self, prob, W):
        L = prob.L
        one = np.zeros(2 * L * L)
        two = np.zeros(4 * L ** 4)
        self.lib.sbo_rdm(ctypes.c_int(L), _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta),
                         ctypes.c_size_t(prob.nb), _d(np.ascontiguousarray(W, dtype=np.float64)), _d(one), _d(two))
        return one, two

    def occupation(self, prob, W):
        out = np.zeros(2 * prob.L)
        self.lib.sbo_occupation(ctypes.c_int(prob.L), _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta),
                                ctypes.c_size_t(prob.nb), _d(np.ascontiguousarray(W, dtype=np.float64)), _d(out))
        return out

    def carryover(self, W, na, nb, ratio=0.0, threshold=0.01):
        order = np.zeros(max(na, 1), np.uint64)
        trunc = ctypes.c_double(0.0)
        n = self.lib.sbo_carryover(_d(np.ascontiguousarray(W, dtype=np.float64)), ctypes.c_size_t(na),
                                   ctypes.c_size_t(nb), ctypes.c_double(ratio), ctypes.c_double(threshold),
                                   _u(order), ctypes.byref(trunc))
        return order[:n], trunc.value

    def rdm_energy(self, prob, one, two):
        return self.lib.sbo_rdm_energy(ctypes.c_int(prob.L), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri),
                                       _d(one), _d(two))


class Ref:
    """The unmodified reference, compiled by oracle/Makefile."""

    def __init__(self, path: str = REF_SO):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_connectivity.restype = ctypes.c_longlong
        L.ref_sigma_sample.restype = ctypes.c_double
        L.ref_davidson.restype = ctypes.c_double
        L.ref_tpb_diag.restype = ctypes.c_longlong
        L.ref_tpb_diag_files.restype = ctypes.c_longlong
        L.ref_load_alpha_dets.restype = ctypes.c_longlong
        L.ref_fcidump_roundtrip.restype = ctypes.c_int

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def _ham(self, prob):
        return (ctypes.c_int(prob.L), ctypes.c_int(prob.nelec), ctypes.c_double(prob.I0), _d(prob.h), _d(prob.eri))

    def connectivity(self, alpha, beta, L, bit_length=20):
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        b = np.ascontiguousarray(beta, dtype=np.uint64)
        out = [np.zeros(len(a), np.uint64), np.zeros(len(a), np.uint64), np.zeros(len(b), np.uint64), np.zeros(len(b), np.uint64)]
        n = self.lib.ref_connectivity(_u(a), ctypes.c_size_t(len(a)), _u(b), ctypes.c_size_t(len(b)), ctypes.c_int(L),
                                      ctypes.c_int(bit_length), *[_u(x) for x in out], None, ctypes.c_longlong(0))
        flat = np.zeros(max(n, 1), np.uint64)
        self.lib.ref_connectivity(_u(a), ctypes.c_size_t(len(a)), _u(b), ctypes.c_size_t(len(b)), ctypes.c_int(L),
                                  ctypes.c_int(bit_length), *[_u(x) for x in out], _u(flat), ctypes.c_longlong(n))
        return out, flat[:n]

    def hij(self, prob, bra_a, bra_b, ket_a, ket_b, bit_length=20):
        n = len(bra_a)
        out = np.zeros(n)
        od = np.zeros(n, np.uint64)
        arrs = [np.ascontiguousarray(x, dtype=np.uint64) for x in (bra_a, bra_b, ket_a, ket_b)]
        self.lib.ref_hij(*self._ham(prob), ctypes.c_int(bit_length), ctypes.c_size_t(n), *[_u(x) for x in arrs], _d(out), _u(od))
        return out, od

    def diag_terms(self, prob, bit_length=20):
        out = np.zeros(prob.na * prob.nb)
        self.lib.ref_diag_terms(*self._ham(prob), ctypes.c_int(bit_length), _u(prob.alpha), ctypes.c_size_t(prob.na),
                                _u(prob.beta), ctypes.c_size_t(prob.nb), _d(out))
        return out

    def sigma(self, prob, C, bit_length=20):
        C = np.ascontiguousarray(C, dtype=np.float64)
        out = np.zeros_like(C)
        self.lib.ref_sigma(*self._ham(prob), ctypes.c_int(bit_length), _u(prob.alpha), ctypes.c_size_t(prob.na),
                           _u(prob.beta), ctypes.c_size_t(prob.nb), _d(C), _d(out))
        return out

    def sigma_sample(self, prob, C, rows, threads=0, bit_length=20):
        C = np.ascontiguousarray(C, dtype=np.float64)
        pairs = ctypes.c_double(0.0)
        S = np.zeros(rows * prob.nb)
        t = self.lib.ref_sigma_sample(*self._ham(prob), ctypes.c_int(bit_length), _u(prob.alpha), ctypes.c_size_t(prob.na),
                                      _u(prob.beta), ctypes.c_size_t(prob.nb), _d(C), _d(S), ctypes.c_size_t(rows),
                                      ctypes.c_int(threads), ctypes.byref(pairs))
        return t, pairs.value, S

    def sigma_rows(self, prob, C, row0, rows, threads=0, bit_length=20):
        """Off-diagonal part of the reference mult on the bra alpha rows
        [row0, row0 + rows) with all kets (ref_sigma_sample_range: the
        diagonal is zero there): rows x nb values, row-major."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        S = np.zeros(rows * prob.nb)
        sec = np.zeros(1)
        pairs = ctypes.c_double(0.0)
        self.lib.ref_sigma_sample_range.restype = ctypes.c_double
        self.lib.ref_sigma_sample_range(*self._ham(prob), ctypes.c_int(bit_length), _u(prob.alpha),
                                        ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb), _d(C),
                                        _d(S), ctypes.c_size_t(row0), ctypes.c_size_t(rows), ctypes.c_int(threads),
                                        ctypes.c_int(1), _d(sec), ctypes.byref(pairs))
        return S

    def rdm(self, prob, W, bit_length=20):
        L = prob.L
        one = np.zeros(2 * L * L)
        two = np.zeros(4 * L ** 4)
        self.lib.ref_rdm(ctypes.c_int(L), _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta), ctypes.c_size_t(prob.nb),
                         ctypes.c_int(bit_length), _d(np.ascontiguousarray(W, dtype=np.float64)), _d(one), _d(two))
        return one, two

    def davidson(self, prob, max_it=1, max_nb=10, eps=1e-4, bit_length=20):
        W = np.zeros(prob.na * prob.nb)
        E = self.lib.ref_davidson(*self._ham(prob), ctypes.c_int(bit_length), _u(prob.alpha), ctypes.c_size_t(prob.na),
                                  _u(prob.beta), ctypes.c_size_t(prob.nb), ctypes.c_int(max_it), ctypes.c_int(max_nb),
                                  ctypes.c_double(eps), _d(W))
        return E, W

    def tpb_diag(self, prob, max_it=1, max_nb=10, eps=1e-4, do_rdm=0, ratio=0.0, threshold=0.01, bit_length=20):
        L = prob.L
        E = ctypes.c_double(0.0)
        dens = np.zeros(2 * L)
        carry = np.zeros(prob.na + 1, np.uint64)
        one = np.zeros(2 * L * L) if do_rdm else None
        two = np.zeros(4 * L ** 4) if do_rdm else None
        n = self.lib.ref_tpb_diag(*self._ham(prob), _u(prob.alpha), ctypes.c_size_t(prob.na), _u(prob.beta),
                                  ctypes.c_size_t(prob.nb), ctypes.c_int(bit_length), ctypes.c_int(max_it),
                                  ctypes.c_int(max_nb), ctypes.c_double(eps), ctypes.c_int(do_rdm),
                                  ctypes.c_double(ratio), ctypes.c_double(threshold), ctypes.byref(E), _d(dens),
                                  _u(carry), ctypes.c_longlong(len(carry)), _d(one), _d(two))
        return dict(energy=E.value, density=dens, carryover=carry[: min(n, len(carry))], one=one, two=two)

    def tpb_diag_files(self, fcidump, adetfile, L, max_it=1, max_nb=10, eps=1e-4, do_rdm=0, ratio=0.0,
                       threshold=0.01, bit_length=20, max_strings=100000):
        E = ctypes.c_double(0.0)
        dens = np.zeros(2 * L)
        carry = np.zeros(max_strings, np.uint64)
        one = np.zeros(2 * L * L) if do_rdm else None
        two = np.zeros(4 * L ** 4) if do_rdm else None
        n = self.lib.ref_tpb_diag_files(fcidump.encode(), adetfile.encode(), ctypes.c_int(bit_length), ctypes.c_int(max_it),
                                        ctypes.c_int(max_nb), ctypes.c_double(eps), ctypes.c_int(do_rdm),
                                        ctypes.c_double(ratio), ctypes.c_double(threshold), ctypes.byref(E), _d(dens),
                                        ctypes.c_int(2 * L), _u(carry), ctypes.c_longlong(max_strings), _d(one), _d(two))
        return dict(energy=E.value, density=dens, carryover=carry[:n], one=one, two=two)

    def load_alpha_dets(self, path, L, bit_length=20, cap=200000):
        out = np.zeros(cap, np.uint64)
        n = self.lib.ref_load_alpha_dets(path.encode(), ctypes.c_int(L), ctypes.c_int(bit_length), _u(out), ctypes.c_longlong(cap))
        return out[:n]

    def fcidump_roundtrip(self, path):
        Lv, Nv, I0 = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0.0)
        n = self.lib.ref_fcidump_roundtrip(path.encode(), ctypes.byref(Lv), ctypes.byref(Nv), ctypes.byref(I0), None, None,
                                           ctypes.c_longlong(0))
        L = Lv.value
        h = np.zeros(L * L)
        eri = np.zeros(n)
        self.lib.ref_fcidump_roundtrip(path.encode(), ctypes.byref(Lv), ctypes.byref(Nv), ctypes.byref(I0), _d(h), _d(eri),
                                       ctypes.c_longlong(n))
        return L, Nv.value, I0.value, h, eri

    def save_wavefunction(self, file, alpha, beta, L, W, bit_length=20):
        """Reference SaveWavefunction (restart.h:20-67): writes file + '000000'."""
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        b = np.ascontiguousarray(beta, dtype=np.uint64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        assert W.size == len(a) * len(b)
        self.lib.ref_save_wavefunction(file.encode(), _u(a), ctypes.c_size_t(len(a)), _u(b), ctypes.c_size_t(len(b)),
                                       ctypes.c_int(L), ctypes.c_int(bit_length), _d(W))

    def load_wavefunction(self, file, alpha, beta, L, bit_length=20):
        """Reference LoadWavefunction (restart.h:414-657) onto the basis (alpha, beta)."""
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        b = np.ascontiguousarray(beta, dtype=np.uint64)
        W = np.zeros(len(a) * len(b))
        rc = self.lib.ref_load_wavefunction(file.encode(), _u(a), ctypes.c_size_t(len(a)), _u(b),
                                            ctypes.c_size_t(len(b)), ctypes.c_int(L), ctypes.c_int(bit_length), _d(W))
        if rc != 0:
            raise RuntimeError("reference LoadWavefunction returned a vector of the wrong size")
        return W
