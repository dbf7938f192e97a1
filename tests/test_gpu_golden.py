"""CUDA path (C-ABI) against the reference's golden outputs (tests/golden).

Connectivity bit-exact; diagonal and sigma within 1e-12 relative; Davidson
energy within 1e-9 Ha; 1-/2-RDM within 1e-8; density within 1e-8; carry-over
strings as a set.
"""
import os

import numpy as np
import pytest

import sbdx
from sbdx import synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    g = dict(np.load(os.path.join(GOLD, f"{name}.npz")))
    prob = synth.Problem(L=int(g["L"]), nelec=int(g["nelec"]), I0=float(g["I0"]), h=g["h"], eri=g["eri"],
                         alpha=g["alpha"].astype(np.uint64), beta=g["beta"].astype(np.uint64))
    return prob, g


@pytest.mark.parametrize("name", ["small_a", "small_b", "small_c"])
def test_cuda_matches_reference_golden(name):
    prob, g = load(name)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        sa, da, ia = ctx.connectivity(0)
        sb, db, ib = ctx.connectivity(1)
        assert np.array_equal(sa, g["a_slen"]) and np.array_equal(da, g["a_dlen"])
        assert np.array_equal(sb, g["b_slen"]) and np.array_equal(db, g["b_dlen"])
        assert np.array_equal(np.concatenate([ia, ib]), g["conn_flat"])
        hii = ctx.diag_terms()
        assert np.abs(hii - g["hii"]).max() <= 1e-12 * np.abs(g["hii"]).max()
        S = ctx.sigma(g["C"])
        assert np.abs(S - g["S"]).max() <= 1e-12 * np.abs(g["S"]).max()
        info, W = ctx.davidson(max_it=6, max_nb=10, eps=1e-10)
        assert abs(info.energy - float(g["E"])) < 1e-9
        one, two = ctx.rdm(g["W"], two="two" in g)
        assert np.abs(one - g["one"]).max() < 1e-8
        if "two" in g:
            assert np.abs(two - g["two"]).max() < 1e-8
        dens = ctx.occupation(W)
        assert np.abs(dens - g["diag_density"]).max() < 1e-8
        wa = ctx.alpha_weights(W)
    order = np.argsort(-wa, kind="stable")
    cum = np.cumsum(wa[order])
    kept = min(int(np.searchsorted(cum, 1.0 - 0.01, side="right")) + 1, len(wa))
    assert set(prob.alpha[order[:kept]].tolist()) == set(g["diag_carry"].tolist())


def test_cfg1_workload_against_reference():
    """The CPU-runnable workload (L=24, 5+5 electrons, 400 x 400 strings)
    against the compiled reference: one sigma of a seeded vector through 8
    seeded projections and 256 seeded entries (1e-12 relative to |S|), the
    plain FP64 Davidson energy (max subspace 16, tolerance 1e-8; 1e-9 Ha) and
    the mixed-precision one (1e-8 Ha)."""
    g = dict(np.load(os.path.join(GOLD, "cfg1.npz")))
    prob = synth.config("cfg1")
    C = np.random.default_rng(2024).standard_normal(prob.D)
    R = np.random.default_rng(2025).standard_normal((8, prob.D))
    norm = float(g["norm"])
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        S = ctx.sigma(C)
        assert abs(np.linalg.norm(S) - norm) <= 1e-12 * norm
        assert np.abs(S[g["idx"]] - g["entries"]).max() <= 1e-12 * norm
        assert np.abs(R @ S - g["proj"]).max() <= 1e-12 * norm * np.sqrt(prob.D)
        info, _ = ctx.davidson(max_it=20, max_nb=16, eps=1e-8)
        assert info.converged == 1 and abs(info.energy - float(g["E"])) < 1e-9
        info32, _ = ctx.davidson(max_it=20, max_nb=16, eps=1e-8, precision=sbdx.SBDX_FP32)
        assert info32.converged == 1 and abs(info32.energy - float(g["E"])) < 1e-8


def test_cfg2_rows_against_reference():
    """The headline workload (L=58, 7+7 electrons, 8000 x 8000 strings):
    the FP64 sigma of a seeded 64 M-element vector, off-diagonal part of 16
    bra alpha rows from the middle of the list, against the reference mult
    on those rows (seeded projections and entries, 1e-12 relative to the
    rows' norm)."""
    g = dict(np.load(os.path.join(GOLD, "cfg2_rows.npz")))
    row0, rows = int(g["row0"]), int(g["rows"])
    prob = synth.config("cfg2")
    C = np.random.default_rng(2027).standard_normal(prob.D)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        S = ctx.sigma(C)
        hii = ctx.diag_terms()
    blk = slice(row0 * prob.nb, (row0 + rows) * prob.nb)
    off = S[blk] - hii[blk] * C[blk]
    del S, hii, C
    norm = float(g["norm"])
    R = np.random.default_rng(2028).standard_normal((8, off.size))
    assert abs(np.linalg.norm(off) - norm) <= 1e-12 * norm
    assert np.abs(off[g["idx"]] - g["entries"]).max() <= 1e-12 * norm
    assert np.abs(R @ off - g["proj"]).max() <= 1e-12 * norm * np.sqrt(off.size)


def test_cfg4_rdm_against_reference():
    """The differentiation workload (L=32, 6+6 electrons, 2000 x 2000
    strings): 1-/2-RDM of a seeded unit vector against the reference
    Correlation (1-RDM whole, 2-RDM through seeded projections and entries;
    1e-8 max-abs)."""
    g = dict(np.load(os.path.join(GOLD, "cfg4_rdm.npz")))
    prob = synth.config("cfg4")
    W = np.random.default_rng(2030).standard_normal(prob.D)
    W /= np.linalg.norm(W)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        one, two = ctx.rdm(W)
    assert np.abs(one - g["one"]).max() < 1e-8
    assert np.abs(two[g["two_idx"]] - g["two_entries"]).max() < 1e-8
    assert abs(np.linalg.norm(two) - float(g["two_norm"])) < 1e-8
    R = np.random.default_rng(2031).standard_normal((8, two.size))
    assert np.abs(R @ two - g["two_proj"]).max() < 1e-8 * np.sqrt(two.size)


@pytest.mark.parametrize("mol", ["h2o", "n2"])
def test_known_answer_energies_cabi(mol):
    g = dict(np.load(os.path.join(GOLD, f"{mol}_1em3.npz")))
    a = g["alpha"].astype(np.uint64)
    L = int(g["L"])
    file_prob = synth.Problem(L=L, nelec=int(g["nelec"]), I0=float(g["I0_rt"]), h=g["h_rt"], eri=g["eri_rt"],
                              alpha=a, beta=a)
    with sbdx.Context(0) as ctx:
        ctx.load(file_prob)
        info, W = ctx.davidson(max_it=10, max_nb=10, eps=1e-8)
        assert abs(info.energy - float(g["E_file"])) < 1e-9
        assert np.abs(ctx.occupation(W) - g["density_file"]).max() < 1e-8
        one, _ = ctx.rdm(W, two=False)
        assert np.abs(one - g["one_file"]).max() < 1e-8
        ctx.set_integrals(L, float(g["I0"]), g["h"], g["eri"])
        info2, _ = ctx.davidson(max_it=10, max_nb=10, eps=1e-8)
        assert abs(info2.energy - float(g["E_struct"])) < 1e-9
