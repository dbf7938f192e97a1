"""Parity of the CUDA path (through the C-ABI) with the oracle on seeded inputs.

Tolerances: connectivity bit-exact; diagonal and FP64 sigma within 1e-12
relative to max |value|; FP64 Davidson energy within 1e-9 Ha; RDMs within
1e-8 max-abs; FP32-storage sigma within 2e-6 relative.
"""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

PROBLEMS = [
    (10, 3, 2, 40, 30, 7),     # unequal alpha/beta electron counts
    (12, 4, 4, 120, 90, 11),
    (16, 3, 5, 60, 200, 13),
    (24, 5, 5, 150, 150, 17),
    (40, 6, 6, 120, 140, 19),
]


@pytest.fixture(scope="module")
def port():
    return Port()


def _prob(spec):
    L, na_el, nb_el, Na, Nb, seed = spec
    return synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)


@pytest.mark.parametrize("spec", PROBLEMS)
def test_connectivity_bit_exact(spec, port):
    prob = _prob(spec)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        for spin, s in ((0, prob.alpha), (1, prob.beta)):
            sl, dl, idx = ctx.connectivity(spin)
            rsl, rdl, ridx = port.connectivity(s)
            assert np.array_equal(sl, rsl) and np.array_equal(dl, rdl)
            assert np.array_equal(idx, ridx)


@pytest.mark.parametrize("spec", PROBLEMS)
def test_diag_and_sigma_fp64(spec, port):
    prob = _prob(spec)
    rng = np.random.default_rng(1)
    C = rng.standard_normal(prob.D)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        hii = ctx.diag_terms()
        ref_h = port.diag_terms(prob)
        assert np.abs(hii - ref_h).max() <= 1e-12 * np.abs(ref_h).max()
        S = ctx.sigma(C)
        ref = port.sigma(prob, C)
        assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()


# Workloads whose beta single-excitation lists are very uneven (near-Aufbau
# strings connect to many more strings than the mean), so the balanced
# alpha-beta layout splits lists; the last one needs two CTAs per alpha row.
SKEWED = [("cfg4", 0.25, None), ("cfg1", 1.0, None), ("wide", 20, 17000)]
_SKEWED_CACHE = {}


def _skewed(name, scale, nb):
    if name == "wide":  # few alpha strings x 17000 beta strings (L=20, 6 electrons)
        I0, h, eri = synth.make_integrals(20, 8, seed=91)
        return synth.Problem(L=20, nelec=12, I0=I0, h=h, eri=eri, alpha=synth.sample_strings(20, 6, scale, 92),
                             beta=synth.sample_strings(20, 6, nb, 93))
    return synth.config(name, scale)


@pytest.mark.parametrize("name,scale,nb", SKEWED)
@pytest.mark.parametrize("tuning", [(0, 0), (21, 61), (28, 64), (24, 71), (14, 42)])
def test_sigma_split_lists_and_orderings(name, scale, nb, tuning, port):
    """Default (alpha-first, balanced) and explicit launch codes, including the
    interleaved kernels, against the oracle."""
    key = (name, scale, nb)
    if key not in _SKEWED_CACHE:
        prob = _skewed(name, scale, nb)
        C = np.random.default_rng(3).standard_normal(prob.D)
        _SKEWED_CACHE[key] = (prob, C, port.sigma(prob, C))
    prob, C, ref = _SKEWED_CACHE[key]
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_tuning(*tuning)
        S = ctx.sigma(C)
    assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()


def test_sigma_fp32_storage(port):
    torch = pytest.importorskip("torch")
    prob = _prob(PROBLEMS[3])
    rng = np.random.default_rng(2)
    C = rng.standard_normal(prob.D)
    ref = port.sigma(prob, C.astype(np.float32).astype(np.float64))
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        dC = torch.tensor(C, dtype=torch.float32, device="cuda")
        dS = torch.empty_like(dC)
        ctx.sigma_device(sbdx.SBDX_FP32, dC.data_ptr(), dS.data_ptr())
        torch.cuda.synchronize()
        S = dS.double().cpu().numpy()
    assert np.abs(S - ref).max() <= 2e-6 * np.abs(ref).max()


# Degenerate shapes: one string on a side (no same-spin entries there, one
# output row or column), an empty and a full spin, the 64-orbital limit
# (pair index 2079, masks up to bit 63); odd sizes exercise the padded row
# strides of the alpha-first vectors.
EDGE = [
    ("1xN", (12, 3, 4, 1, 60, 51)),
    ("Nx1", (12, 4, 3, 70, 1, 52)),
    ("1x1", (8, 2, 2, 1, 1, 53)),
    ("no_alpha_electrons", (10, 0, 3, 1, 50, 54)),
    ("full_beta", (9, 3, 9, 40, 1, 55)),
    ("L64", (64, 3, 3, 80, 70, 57)),
    ("L64_unequal", (64, 6, 5, 121, 93, 58)),
]


@pytest.mark.parametrize("name,spec", EDGE)
def test_edge_shapes(name, spec, port):
    torch = pytest.importorskip("torch")
    prob = _prob(spec)
    C = np.random.default_rng(5).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    ref32 = port.sigma(prob, C.astype(np.float32).astype(np.float64))
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        for spin, strings in ((0, prob.alpha), (1, prob.beta)):
            sl, dl, idx = ctx.connectivity(spin)
            rsl, rdl, ridx = port.connectivity(strings)
            assert np.array_equal(sl, rsl) and np.array_equal(dl, rdl) and np.array_equal(idx, ridx)
        hii = ctx.diag_terms()
        ref_h = port.diag_terms(prob)
        assert np.abs(hii - ref_h).max() <= 1e-12 * np.abs(ref_h).max()
        S = ctx.sigma(C)
        assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()
        dC = torch.tensor(C, dtype=torch.float32, device="cuda")
        dS = torch.empty_like(dC)
        ctx.sigma_device(sbdx.SBDX_FP32, dC.data_ptr(), dS.data_ptr())
        torch.cuda.synchronize()
        S32 = dS.double().cpu().numpy()
        assert np.abs(S32 - ref32).max() <= 2e-6 * np.abs(ref32).max()


@pytest.mark.parametrize("spec", PROBLEMS + [e[1] for e in EDGE])
def test_stored_hamiltonian_sigma(spec, port):
    """The stored Hamiltonian (method 1): its product equals the oracle's
    sigma (1e-12 relative); releasing it returns to the on-the-fly kernels;
    the element count is the reference's per-row count (same-spin lists of
    the row's alpha and beta strings plus singles x singles)."""
    prob = _prob(spec)
    C = np.random.default_rng(6).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        nnz = ctx.build_hamiltonian()
        sa, da, _ = ctx.connectivity(0)
        sb, db, _ = ctx.connectivity(1)
        na_e, nb_e = (sa + da).astype(np.int64), (sb + db).astype(np.int64)
        expect = len(prob.beta) * na_e.sum() + len(prob.alpha) * nb_e.sum() + \
            int(sa.astype(np.int64).sum()) * int(sb.astype(np.int64).sum())
        assert nnz == expect
        S = ctx.sigma(C)
        assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()
        ctx.release_hamiltonian()
        S2 = ctx.sigma(C)
        assert np.abs(S2 - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("spec", PROBLEMS[1:4])
def test_stored_hamiltonian_davidson(spec, port):
    """FP64 Davidson on the stored matrix: the oracle's energy (1e-9 Ha) and
    the on-the-fly solve's."""
    prob = _prob(spec)
    E_ref, _, _ = port.davidson(prob, max_it=6, max_nb=10, eps=1e-9)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_hamiltonian()
        info, W = ctx.davidson(max_it=6, max_nb=10, eps=1e-9)
    assert abs(info.energy - E_ref) < 1e-9


@pytest.mark.parametrize("spec", PROBLEMS[1:4])
def test_davidson_fp64_energy(spec, port):
    prob = _prob(spec)
    E_ref, W_ref, nsig = port.davidson(prob, max_it=6, max_nb=10, eps=1e-9)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W = ctx.davidson(max_it=6, max_nb=10, eps=1e-9)
    assert abs(info.energy - E_ref) < 1e-9
    assert abs(abs(np.dot(W, W_ref)) - 1.0) < 1e-8


@pytest.mark.parametrize("spec", PROBLEMS[1:4])
def test_davidson_mixed_matches_fp64(spec, port):
    prob = _prob(spec)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        i64, W64 = ctx.davidson(max_it=10, max_nb=12, eps=1e-8)
        i32, W32 = ctx.davidson(max_it=10, max_nb=12, eps=1e-8, precision=sbdx.SBDX_FP32)
    assert i32.converged == 1
    assert abs(i32.energy - i64.energy) < 1e-8


@pytest.mark.parametrize("spec", PROBLEMS[:4])
def test_rdm_matches_oracle(spec, port):
    prob = _prob(spec)
    E, W, _ = port.davidson(prob, max_it=4, max_nb=10, eps=1e-8)
    one_r, two_r = port.rdm(prob, W)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        one, two = ctx.rdm(W)
        dens = ctx.occupation(W)
        wa = ctx.alpha_weights(W)
    assert np.abs(one - one_r).max() < 1e-8
    assert np.abs(two - two_r).max() < 1e-8
    assert np.abs(dens - port.occupation(prob, W)).max() < 1e-12
    Wm = W.reshape(prob.na, prob.nb)
    assert np.abs(wa - (Wm ** 2).sum(1)).max() < 1e-12
    assert abs(port.rdm_energy(prob, one, two) - E) < 1e-9
