"""Generate the golden fixtures of the parity tests from the compiled reference.

Run in a container where the reference tree is mounted and oracle/_ref has
been built (make -C oracle ref):

    python tests/golden/make_golden.py

Every array in the fixtures is an output of the UNMODIFIED reference headers
(walkup/sbd-ykt), driven through oracle/ref_driver.cc:
  * small_*.npz : seeded synthetic problems -- connectivity lists
                  (GenerateExcitation/MakeSmartHelper), matrix elements of
                  sampled determinant pairs (Hij), diagonal (makeQChamDiagTerms),
                  one sigma (mult), Davidson energy and vector, 1-/2-RDM
                  (Correlation), and the tpb::diag outputs (energy, density,
                  carry-over strings) on the struct path;
  * cfg1.npz : the CPU-runnable synthetic workload (400 x 400 strings,
                  L = 24): the tpb::diag energy and density, and seeded
                  projections and entries of one sigma (mult);
  * cfg2_rows.npz : the headline workload (8000 x 8000 strings, L = 58):
                  the reference mult on 16 bra alpha rows of a seeded vector,
                  as seeded projections and entries;
  * cfg4_rdm.npz : the differentiation workload (2000 x 2000 strings,
                  L = 32): the Correlation 1-/2-RDM of a seeded unit vector;
  * h2o_1em3.npz / n2_1em3.npz : the reference's own known-answer inputs
                  (data/h2o, data/n2 with the 1e-3 string files) as parsed by
                  LoadFCIDump/LoadAlphaDets, the integrals after the file path's
                  text round trip, and the energies of both entry points.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "sbd-ykt_b200")]

from oracle import Ref, reference_root  # noqa: E402
from sbdx import synth  # noqa: E402

REF = reference_root()  # $SBD_REFERENCE, else the mounted tree

SMALL = {
    # name: (L, n_alpha, n_beta, Na, Nb, seed)
    "small_a": (10, 3, 2, 40, 30, 7),
    "small_b": (14, 4, 4, 90, 70, 21),
    "small_c": (20, 3, 5, 50, 120, 33),
}


def small(ref: Ref, name, spec):
    L, na_el, nb_el, Na, Nb, seed = spec
    prob = synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)
    (asl, adl, bsl, bdl), flat = ref.connectivity(prob.alpha, prob.beta, L)
    rng = np.random.default_rng(seed)
    n = 4000
    ia = rng.integers(0, prob.na, n)
    ib = rng.integers(0, prob.nb, n)
    ja = rng.integers(0, prob.na, n)
    jb = rng.integers(0, prob.nb, n)
    ja[: n // 3] = ia[: n // 3]
    jb[n // 3: 2 * n // 3] = ib[n // 3: 2 * n // 3]
    hij, od = ref.hij(prob, prob.alpha[ia], prob.beta[ib], prob.alpha[ja], prob.beta[jb])
    hii = ref.diag_terms(prob)
    C = rng.standard_normal(prob.D)
    S = ref.sigma(prob, C)
    E, W = ref.davidson(prob, max_it=6, max_nb=10, eps=1e-10)
    one, two = ref.rdm(prob, W)
    d = ref.tpb_diag(prob, max_it=6, max_nb=10, eps=1e-10, do_rdm=0, ratio=0.0, threshold=0.01)
    d2 = ref.tpb_diag(prob, max_it=6, max_nb=10, eps=1e-10, do_rdm=0, ratio=0.5, threshold=0.01)
    extra = {"two": two} if L <= 14 else {}  # the 4*L^4 2-RDM only for the small orbital counts
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"), L=L, nelec=prob.nelec, I0=prob.I0, h=prob.h, eri=prob.eri,
        alpha=prob.alpha, beta=prob.beta, a_slen=asl, a_dlen=adl, b_slen=bsl, b_dlen=bdl, conn_flat=flat,
        pair_ia=ia, pair_ib=ib, pair_ja=ja, pair_jb=jb, hij=hij, orb_diff=od, hii=hii, C=C, S=S, E=E, W=W,
        one=one, diag_energy=d["energy"], diag_density=d["density"], diag_carry=d["carryover"],
        diag_carry_ratio=d2["carryover"], **extra)
    print(name, prob.na, prob.nb, "E", E)


def kat(ref: Ref, mol, fcidump, adet, L):
    La, N, I0r, hr, erir = ref.fcidump_roundtrip(fcidump)
    assert La == L
    alpha = ref.load_alpha_dets(adet, L)
    # exact doubles as written in the file (no round trip), for the struct path
    h = np.zeros((L, L))
    eri = np.zeros(len(erir))
    I0 = 0.0
    with open(fcidump) as f:
        for line in f:
            parts = line.split()
            if len(parts) != 5 or "&" in line or "=" in line:
                continue
            try:
                v = float(parts[0])
                i, j, k, l = (int(x) for x in parts[1:])
            except ValueError:
                continue
            if i == j == k == l == 0:
                I0 = v
            elif k == 0 and l == 0:
                h[i - 1, j - 1] = h[j - 1, i - 1] = v
            else:
                eri[synth.eri_index(i - 1, j - 1, k - 1, l - 1)] = v
    file_path = ref.tpb_diag_files(fcidump, adet, L, max_it=10, max_nb=10, eps=1e-8, do_rdm=1)
    prob = synth.Problem(L=L, nelec=N, I0=I0, h=h.reshape(-1), eri=eri, alpha=alpha, beta=alpha.copy())
    struct = ref.tpb_diag(prob, max_it=10, max_nb=10, eps=1e-8, do_rdm=0)
    np.savez_compressed(
        os.path.join(HERE, f"{mol}_1em3.npz"), L=L, nelec=N, I0=I0, h=h.reshape(-1), eri=eri, alpha=alpha,
        I0_rt=I0r, h_rt=hr, eri_rt=erir, E_file=file_path["energy"], density_file=file_path["density"],
        carry_file=file_path["carryover"], one_file=file_path["one"], E_struct=struct["energy"])
    print(mol, len(alpha), "E_file", file_path["energy"], "E_struct", struct["energy"])


def cfg1(ref: Ref):
    """The CPU-runnable plain-FP64 workload (L=24, 5+5 electrons, 400 x 400
    strings): tpb::diag energy (max subspace 16, tolerance 1e-8) and one
    sigma of a seeded vector, kept as size-independent checks (seeded
    projections and seeded entries) so that the fixture stays small."""
    prob = synth.config("cfg1")
    rng = np.random.default_rng(2024)
    C = rng.standard_normal(prob.D)
    S = ref.sigma(prob, C)
    R = np.random.default_rng(2025).standard_normal((8, prob.D))
    idx = np.random.default_rng(2026).choice(prob.D, 256, replace=False)
    struct = ref.tpb_diag(prob, max_it=20, max_nb=16, eps=1e-8, do_rdm=0)
    np.savez_compressed(os.path.join(HERE, "cfg1.npz"), proj=R @ S, norm=np.linalg.norm(S), idx=idx, entries=S[idx],
                        E=struct["energy"], density=struct["density"])
    print("cfg1", prob.D, "E", struct["energy"])


def cfg2_rows(ref: Ref, row0=3992, rows=16):
    """The headline workload (L=58, 7+7 electrons, 8000 x 8000 strings, 64 M
    determinants): the reference mult on bra alpha rows [row0, row0 + rows)
    of a seeded vector (off-diagonal part; a whole sigma takes about an hour
    on the host), kept as seeded projections and entries of those rows."""
    prob = synth.config("cfg2")
    C = np.random.default_rng(2027).standard_normal(prob.D)
    S = ref.sigma_rows(prob, C, row0, rows)
    R = np.random.default_rng(2028).standard_normal((8, S.size))
    idx = np.random.default_rng(2029).choice(S.size, 256, replace=False)
    np.savez_compressed(os.path.join(HERE, "cfg2_rows.npz"), row0=row0, rows=rows, proj=R @ S,
                        norm=np.linalg.norm(S), idx=idx, entries=S[idx])
    print("cfg2 rows", row0, rows, "norm", np.linalg.norm(S))


def cfg4_rdm(ref: Ref):
    """The differentiation workload (L=32, 6+6 electrons, 2000 x 2000
    strings): the reference Correlation 1-/2-RDM of a seeded unit vector
    (the RDMs are bilinear in W, so any vector tests the kernels): the
    1-RDM whole, the 2-RDM as seeded projections and entries."""
    prob = synth.config("cfg4")
    W = np.random.default_rng(2030).standard_normal(prob.D)
    W /= np.linalg.norm(W)
    one, two = ref.rdm(prob, W)
    R = np.random.default_rng(2031).standard_normal((8, two.size))
    idx = np.random.default_rng(2032).choice(two.size, 512, replace=False)
    np.savez_compressed(os.path.join(HERE, "cfg4_rdm.npz"), one=one, two_norm=np.linalg.norm(two), two_proj=R @ two,
                        two_idx=idx, two_entries=two[idx])
    print("cfg4 rdm", np.abs(one).max(), np.linalg.norm(two))


def main():
    if not Ref.available():
        raise SystemExit("oracle/_ref/libsbdref.so missing: run make -C oracle ref")
    ref = Ref()
    for name, spec in SMALL.items():
        small(ref, name, spec)
    cfg1(ref)
    cfg2_rows(ref)
    cfg4_rdm(ref)
    kat(ref, "h2o", f"{REF}/data/h2o/fcidump.txt", f"{REF}/data/h2o/h2o-1em3-alpha.txt", 24)
    kat(ref, "n2", f"{REF}/data/n2/fcidump.txt", f"{REF}/data/n2/1em3-alpha.txt", 18)


if __name__ == "__main__":
    main()
