"""Seeded synthetic workloads for the sbd tpb selected-CI path.

The workloads follow the integral and string laws stated for the benchmark
configurations (there is no public dataset for this path):

* one-electron h: symmetric, diagonal linearly spaced from -20 to +2 Ha,
  off-diagonal N(0, 0.05^2);
* two-electron (pq|rs) = sum_{k<K} L^k_pq L^k_rs with symmetric
  L^k_pq ~ N(0, 0.1^2 / (1 + |p - q|)) (8-fold symmetric and PSD);
* core energy I0 = 9.0;
* strings: excitation rank k from the Aufbau string with P(k) ~ exp(-k),
  k <= min(n, L - n), holes uniform in the occupied set and particles uniform
  in the virtuals; draws repeat until N unique strings are found (Aufbau is
  always included); the set is sorted ascending so index 0 is Aufbau, the
  Hartree-Fock start of the reference (chemistry/tpb/davidson.h:130-133).

Integrals are returned as exact doubles (the struct path of tpb::diag) and can
be written as an FCIDUMP text file (the file path).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


def npair(L: int) -> int:
    return L * (L + 1) // 2


def neri(L: int) -> int:
    P = npair(L)
    return P * (P + 1) // 2


def pair_index(p, q):
    p, q = np.maximum(p, q), np.minimum(p, q)
    return p * (p + 1) // 2 + q


def eri_index(p, q, r, s):
    a = pair_index(p, q)
    b = pair_index(r, s)
    return pair_index(a, b)


@dataclasses.dataclass
class Problem:
    L: int
    nelec: int
    I0: float
    h: np.ndarray       # L*L, row-major
    eri: np.ndarray     # 8-fold packed
    alpha: np.ndarray   # uint64 strings
    beta: np.ndarray    # uint64 strings
    name: str = ""

    @property
    def na(self) -> int:
        return int(len(self.alpha))

    @property
    def nb(self) -> int:
        return int(len(self.beta))

    @property
    def D(self) -> int:
        return self.na * self.nb

    def with_strings(self, alpha, beta):
        return dataclasses.replace(self, alpha=np.ascontiguousarray(alpha, dtype=np.uint64),
                                   beta=np.ascontiguousarray(beta, dtype=np.uint64))


def make_integrals(L: int, K: int, seed: int, I0: float = 9.0):
    """One- and two-electron integrals of the synthetic law (exact doubles)."""
    rng = np.random.default_rng(seed)
    h = rng.normal(0.0, 0.05, size=(L, L))
    h = np.triu(h, 1)
    h = h + h.T
    h[np.diag_indices(L)] = np.linspace(-20.0, 2.0, L)
    p, q = np.tril_indices(L)  # p >= q, row-major over packed pair index
    order = np.argsort(pair_index(p, q))
    p, q = p[order], q[order]
    std = 0.1 / np.sqrt(1.0 + np.abs(p - q))
    Lk = rng.normal(size=(K, len(p))) * std[None, :]   # L^k on packed pairs
    V = Lk.T @ Lk                                      # (pq|rs) over packed pairs
    P = len(p)
    a, b = np.tril_indices(P)
    eri = np.zeros(neri(L))
    eri[pair_index(a, b)] = V[a, b]
    return float(I0), np.ascontiguousarray(h.reshape(-1)), eri


def sample_strings(L: int, n: int, N: int, seed: int, batch: int = 65536) -> np.ndarray:
    """N unique strings of n electrons in L orbitals, sorted ascending."""
    if L > 64:
        raise ValueError("L must be <= 64")
    total = math.comb(L, n)
    if N > total:
        raise ValueError(f"only {total} strings exist for L={L}, n={n}")
    rng = np.random.default_rng(seed)
    kmax = min(n, L - n)
    pk = np.exp(-np.arange(kmax + 1, dtype=np.float64))
    pk /= pk.sum()
    aufbau = (1 << n) - 1
    seen = {aufbau: 0}
    found = [aufbau]
    while len(found) < N:
        ks = rng.choice(kmax + 1, size=batch, p=pk)
        hk = np.argsort(rng.random((batch, n)), axis=1)
        pkk = np.argsort(rng.random((batch, L - n)), axis=1) + n
        for t in range(batch):
            k = int(ks[t])
            x = aufbau
            for j in range(k):
                x &= ~(1 << int(hk[t, j]))
                x |= 1 << int(pkk[t, j])
            if x not in seen:
                seen[x] = len(found)
                found.append(x)
                if len(found) == N:
                    break
    out = np.array(sorted(found), dtype=np.uint64)
    return out


# name -> (L, n, K, Na, Nb, seed_integrals, seed_alpha, seed_beta, max_nb, tol)
CONFIGS = {
    "cfg1": (24, 5, 48, 400, 400, 1001, 1011, 1012, 16, 1e-8),
    "cfg2": (58, 7, 96, 8000, 8000, 2001, 2011, 2012, 12, 1e-8),
    "cfg3": (58, 7, 96, 20000, 20000, 2001, 3011, 3012, 12, 1e-8),
    "cfg4": (32, 6, 96, 2000, 2000, 4001, 4011, 4012, 12, 1e-10),
}


def config(name: str, scale: float = 1.0) -> Problem:
    """A named benchmark workload; `scale` shrinks the string counts (tests)."""
    L, n, K, Na, Nb, si, sa, sb, _, _ = CONFIGS[name]
    I0, h, eri = make_integrals(L, K, si)
    na = max(2, int(round(Na * scale)))
    nb = max(2, int(round(Nb * scale)))
    a = sample_strings(L, n, na, sa)
    b = sample_strings(L, n, nb, sb)
    return Problem(L=L, nelec=2 * n, I0=I0, h=h, eri=eri, alpha=a, beta=b, name=name)


def batched_config(n_sub: int = 64, seed: int = 5001, lo: int = 200, hi: int = 4000, scale: float = 1.0):
    """64 subspaces sharing one Hamiltonian (L=40, n=8), Na and Nb log-uniform."""
    L, n, K = 40, 8, 96
    I0, h, eri = make_integrals(L, K, seed)
    rng = np.random.default_rng(seed + 1)
    subs = []
    for k in range(n_sub):
        na = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) * scale))
        nb = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) * scale))
        na, nb = max(na, 2), max(nb, 2)
        a = sample_strings(L, n, na, seed + 100 + 2 * k)
        b = sample_strings(L, n, nb, seed + 101 + 2 * k)
        subs.append(Problem(L=L, nelec=2 * n, I0=I0, h=h, eri=eri, alpha=a, beta=b, name=f"sub{k}"))
    return subs


def random_problem(L: int, na_el: int, nb_el: int, Na: int, Nb: int, seed: int, K: int = 8) -> Problem:
    """Small random problem (possibly unequal alpha/beta electron counts)."""
    I0, h, eri = make_integrals(L, K, seed)
    a = sample_strings(L, na_el, Na, seed + 1)
    b = sample_strings(L, nb_el, Nb, seed + 2)
    return Problem(L=L, nelec=na_el + nb_el, I0=I0, h=h, eri=eri, alpha=a, beta=b, name=f"rand{seed}")


def det_pairs(slen_a, dlen_a, slen_b, dlen_b) -> dict:
    """det-pairs evaluated by one sigma, counted as the reference enumerates
    them (mult.h:453-578): D diagonal + Nb*sum_a(S+D) + Na*sum_b(S+D)
    + (sum_a S)(sum_b S)."""
    na, nb = len(slen_a), len(slen_b)
    Sa, Da = float(np.sum(slen_a)), float(np.sum(dlen_a))
    Sb, Db = float(np.sum(slen_b)), float(np.sum(dlen_b))
    same = nb * (Sa + Da) + na * (Sb + Db)
    ab = Sa * Sb
    return dict(diagonal=float(na * nb), same_spin=same, alpha_beta=ab, offdiag=same + ab,
                total=float(na * nb) + same + ab, Sa=Sa, Da=Da, Sb=Sb, Db=Db)


def fcidump_text(prob: Problem, fmt: str = "%.17g") -> str:
    """FCIDUMP text with one line per 8-fold ERI class, one-electron lines
    (i >= j), and the core energy, in the order the reference parser accepts
    (framework/fcidump.h:27-139)."""
    L = prob.L
    lines = [f" &FCI NORB={L},NELEC={prob.nelec},MS2=0,", "  ORBSYM=" + "1," * L, "  ISYM=1,", " &END"]
    for p in range(L):
        for q in range(p + 1):
            for r in range(p + 1):
                for s in range(r + 1):
                    if pair_index(r, s) > pair_index(p, q):
                        continue
                    v = prob.eri[eri_index(p, q, r, s)]
                    lines.append((fmt % v) + f" {p + 1} {q + 1} {r + 1} {s + 1}")
    for p in range(L):
        for q in range(p + 1):
            lines.append((fmt % prob.h[p * L + q]) + f" {p + 1} {q + 1} 0 0")
    lines.append((fmt % prob.I0) + " 0 0 0 0")
    return "\n".join(lines) + "\n"


def strings_text(strings, L: int) -> str:
    """Determinant-file text: one '0'/'1' string per line, rightmost char =
    orbital 0 (framework/bit_manipulation.h:135-172)."""
    out = []
    for x in strings:
        x = int(x)
        out.append("".join("1" if (x >> (L - 1 - i)) & 1 else "0" for i in range(L)))
    return "\n".join(out) + "\n"


def write_problem_bin(path: str, prob: Problem):
    """Binary problem file read by the reference CLI (oracle/ref_cli.cc)."""
    with open(path, "wb") as f:
        np.array([prob.L, prob.nelec, prob.na, prob.nb], dtype=np.int64).tofile(f)
        np.array([prob.I0], dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.h, dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.eri, dtype=np.float64).tofile(f)
        np.ascontiguousarray(prob.alpha, dtype=np.uint64).tofile(f)
        np.ascontiguousarray(prob.beta, dtype=np.uint64).tofile(f)
