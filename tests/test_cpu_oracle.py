"""CPU tests: the C restatement (oracle/sbd_oracle.c) against the golden
fixtures produced by the compiled reference (tests/golden/make_golden.py).

Tolerances: connectivity and orbital codes bit-exact; matrix elements and
diagonal 1e-12 absolute; sigma 1e-12 relative; energies 1e-9 Ha; RDMs 1e-9.
"""
import os

import numpy as np
import pytest

from oracle import Port
from sbdx import synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")
SMALL = ["small_a", "small_b", "small_c"]


@pytest.fixture(scope="module")
def port():
    return Port()


def load(name):
    g = dict(np.load(os.path.join(GOLD, f"{name}.npz")))
    prob = synth.Problem(L=int(g["L"]), nelec=int(g["nelec"]), I0=float(g["I0"]), h=g["h"], eri=g["eri"],
                         alpha=g["alpha"].astype(np.uint64), beta=g["beta"].astype(np.uint64))
    return prob, g


@pytest.mark.parametrize("name", SMALL)
def test_connectivity_matches_reference(name, port):
    prob, g = load(name)
    sa, da, ia = port.connectivity(prob.alpha)
    sb, db, ib = port.connectivity(prob.beta)
    assert np.array_equal(sa, g["a_slen"]) and np.array_equal(da, g["a_dlen"])
    assert np.array_equal(sb, g["b_slen"]) and np.array_equal(db, g["b_dlen"])
    assert np.array_equal(np.concatenate([ia, ib]), g["conn_flat"])


@pytest.mark.parametrize("name", SMALL)
def test_matrix_elements_match_reference(name, port):
    prob, g = load(name)
    a, b = prob.alpha, prob.beta
    h = np.array([port.hij(prob, a[x], b[y], a[z], b[w])
                  for x, y, z, w in zip(g["pair_ia"], g["pair_ib"], g["pair_ja"], g["pair_jb"])])
    assert np.abs(h - g["hij"]).max() <= 1e-12
    assert np.count_nonzero(g["hij"]) > 100


@pytest.mark.parametrize("name", SMALL)
def test_diag_and_sigma_match_reference(name, port):
    prob, g = load(name)
    assert np.abs(port.diag_terms(prob) - g["hii"]).max() <= 1e-12
    S = port.sigma(prob, g["C"])
    assert np.abs(S - g["S"]).max() <= 1e-12 * np.abs(g["S"]).max()


@pytest.mark.parametrize("name", SMALL)
def test_davidson_and_rdm_match_reference(name, port):
    prob, g = load(name)
    E, W, _ = port.davidson(prob, max_it=6, max_nb=10, eps=1e-10)
    assert abs(E - float(g["E"])) < 1e-9
    assert abs(abs(np.dot(W, g["W"])) - 1) < 1e-9
    one, two = port.rdm(prob, g["W"])
    assert np.abs(one - g["one"]).max() < 1e-9
    if "two" in g:
        assert np.abs(two - g["two"]).max() < 1e-9
        # the sample driver's energy identity (main.cc:166-216)
        assert abs(port.rdm_energy(prob, one, two) - float(g["E"])) < 1e-9


def test_cfg1_sigma_and_energy_match_reference(port):
    """The CPU-runnable workload (400 x 400 strings, L = 24): the oracle's
    sigma of the seeded vector against the reference's seeded projections
    and entries (1e-12 relative to |S|), and its FP64 Davidson energy (max
    subspace 16, tolerance 1e-8) against the reference's tpb::diag (1e-9 Ha)."""
    g = dict(np.load(os.path.join(GOLD, "cfg1.npz")))
    prob = synth.config("cfg1")
    C = np.random.default_rng(2024).standard_normal(prob.D)
    R = np.random.default_rng(2025).standard_normal((8, prob.D))
    norm = float(g["norm"])
    S = port.sigma(prob, C)
    assert np.abs(S[g["idx"]] - g["entries"]).max() <= 1e-12 * norm
    assert np.abs(R @ S - g["proj"]).max() <= 1e-12 * norm * np.sqrt(prob.D)
    E, _, _ = port.davidson(prob, max_it=20, max_nb=16, eps=1e-8)
    assert abs(E - float(g["E"])) < 1e-9


def test_cfg2_rows_match_reference(port):
    """The headline workload (L=58, 7+7 electrons, 8000 x 8000 strings): the
    oracle's off-diagonal sigma on 16 bra alpha rows of the seeded vector
    against the reference mult on the same rows (seeded projections and
    entries, 1e-12 relative to the rows' norm)."""
    g = dict(np.load(os.path.join(GOLD, "cfg2_rows.npz")))
    prob = synth.config("cfg2")
    C = np.random.default_rng(2027).standard_normal(prob.D)
    S = port.sigma_rows(prob, C, int(g["row0"]), int(g["rows"]))
    del C
    norm = float(g["norm"])
    R = np.random.default_rng(2028).standard_normal((8, S.size))
    assert abs(np.linalg.norm(S) - norm) <= 1e-12 * norm
    assert np.abs(S[g["idx"]] - g["entries"]).max() <= 1e-12 * norm
    assert np.abs(R @ S - g["proj"]).max() <= 1e-12 * norm * np.sqrt(S.size)


@pytest.mark.parametrize("name", SMALL)
def test_tpb_diag_outputs(name, port):
    prob, g = load(name)
    E, W, _ = port.davidson(prob, max_it=6, max_nb=10, eps=1e-10)
    assert abs(E - float(g["diag_energy"])) < 1e-9
    dens = port.occupation(prob, W)
    assert np.abs(dens - g["diag_density"]).max() < 1e-9
    order, _ = port.carryover(W, prob.na, prob.nb, ratio=0.0, threshold=0.01)
    assert set(prob.alpha[order].tolist()) == set(g["diag_carry"].tolist())
    order2, _ = port.carryover(W, prob.na, prob.nb, ratio=0.5)
    assert set(prob.alpha[order2].tolist()) == set(g["diag_carry_ratio"].tolist())


def test_n2_known_answer_file_path(port):
    """n2 6-31G, 1e-3 strings: the file path of tpb::diag (FCIDUMP text round
    trip to 6 significant digits). README: -109.041511 Ha."""
    g = dict(np.load(os.path.join(GOLD, "n2_1em3.npz")))
    L = int(g["L"])
    a = g["alpha"].astype(np.uint64)
    prob = synth.Problem(L=L, nelec=int(g["nelec"]), I0=float(g["I0_rt"]), h=g["h_rt"], eri=g["eri_rt"],
                         alpha=a, beta=a.copy())
    E, W, _ = port.davidson(prob, max_it=10, max_nb=10, eps=1e-8)
    assert abs(E - float(g["E_file"])) < 1e-9
    assert abs(E - (-109.041511)) < 1e-6
    assert np.abs(port.occupation(prob, W) - g["density_file"]).max() < 1e-8


def test_fcidump_roundtrip_rounds_to_six_digits():
    """The file path re-parses integrals printed at 6 significant digits
    (fcidump.h:156-169, 251); the fixture's round-tripped values equal
    float('%.6g' % x) of the exact ones."""
    g = dict(np.load(os.path.join(GOLD, "h2o_1em3.npz")))
    r6 = np.vectorize(lambda x: float("%.6g" % x))
    assert np.array_equal(r6(g["eri"]), g["eri_rt"])
    assert np.array_equal(r6(g["h"]), g["h_rt"])
    assert float("%.6g" % float(g["I0"])) == float(g["I0_rt"])
