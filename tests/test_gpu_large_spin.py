"""More than 65,535 strings on one spin (the reference has no limit; here the
excitation records hold 24-bit string indices).

70,000 strings of 6 electrons in 24 orbitals (a seeded subset of all
134,596) on one spin, the 8 numerically smallest strings of 5 electrons on
the other, both ways round. The oracle's O(n^2) connectivity takes minutes
at this size, so the checks are the size-independent properties of the
product (mult, chemistry/tpb/mult.h:376-632) and of the RDMs (Correlation,
chemistry/tpb/correlation.h:194-444):

- H is symmetric: <x|Hy> = <Hx|y> within 1e-12 of sum |x_i (Hy)_i| for
  seeded x, y (FP64; FP32 storage within 1e-5);
- the order of the strings is a labelling: reversing the large spin's list
  permutes the product's rows or columns the same way (FP64 within 1e-12 of
  max |value|), and leaves the 1-/2-RDM of the permuted vector unchanged
  (within 1e-12). A string index cut to 16 bits anywhere would pair the
  wrong strings in one of the two orders;
- the RDM energy identity (samples/.../main.cc:166-216): E from the 1-/2-RDM
  equals <W|HW> within 1e-9 relative.

The large beta side needs several ket panels in the alpha-beta kernel,
whose records then hold panel-relative positions."""
import itertools

import numpy as np
import pytest
import torch

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

L = 24
N_LARGE = 70000


def _strings(n_el, count, seed=None):
    combos = np.array([sum(1 << i for i in c) for c in itertools.combinations(range(L), n_el)], dtype=np.uint64)
    combos.sort()
    if seed is None:
        return combos[:count].copy()
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(len(combos), size=count, replace=False))
    return combos[pick].copy()


def _problem(large_alpha, reverse=False):
    I0, h, eri = synth.make_integrals(L, 8, 61)
    big = _strings(6, N_LARGE, seed=62)
    if reverse:
        big = big[::-1].copy()
    small = _strings(5, 8)
    a, b = (big, small) if large_alpha else (small, big)
    return synth.Problem(L=L, nelec=11, I0=I0, h=h, eri=eri, alpha=a, beta=b, name="large_spin")


def _flip(v, prob, large_alpha):
    m = v.reshape(prob.na, prob.nb)
    return np.ascontiguousarray(m[::-1, :] if large_alpha else m[:, ::-1]).ravel()


def _sigma32(ctx, x):
    dx = torch.tensor(x, dtype=torch.float32, device="cuda")
    dy = torch.empty_like(dx)
    ctx.sigma_device(sbdx.SBDX_FP32, dx.data_ptr(), dy.data_ptr())
    torch.cuda.synchronize()
    return dx.double().cpu().numpy(), dy.double().cpu().numpy()


@pytest.mark.parametrize("large_alpha", [False, True])
def test_large_spin_sigma_symmetric_and_order_invariant(large_alpha):
    prob = _problem(large_alpha)
    assert max(prob.na, prob.nb) > 65535
    rng = np.random.default_rng(5)
    x, y = rng.standard_normal(prob.D), rng.standard_normal(prob.D)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        Hx, Hy = ctx.sigma(x), ctx.sigma(y)
        assert abs(x @ Hy - Hx @ y) <= 1e-12 * (np.abs(x) @ np.abs(Hy))
        x32, Hx32 = _sigma32(ctx, x)
        y32, Hy32 = _sigma32(ctx, y)
        assert abs(x32 @ Hy32 - Hx32 @ y32) <= 1e-5 * (np.abs(x32) @ np.abs(Hy32))
    rev = _problem(large_alpha, reverse=True)
    with sbdx.Context(0) as ctx:
        ctx.load(rev)
        Hx_rev = ctx.sigma(_flip(x, prob, large_alpha))
    want = _flip(Hx, prob, large_alpha)
    assert np.abs(Hx_rev - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("large_alpha", [False, True])
def test_large_spin_rdm_identity_and_order_invariant(large_alpha):
    prob = _problem(large_alpha)
    W = np.random.default_rng(9).standard_normal(prob.D)
    W /= np.linalg.norm(W)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        one, two = ctx.rdm(W)
        E = W @ ctx.sigma(W)
    assert abs(Port().rdm_energy(prob, one, two) - E) <= 1e-9 * abs(E)
    rev = _problem(large_alpha, reverse=True)
    with sbdx.Context(0) as ctx:
        ctx.load(rev)
        one_r, two_r = ctx.rdm(_flip(W, prob, large_alpha))
    assert np.abs(one_r - one).max() <= 1e-12
    assert np.abs(two_r - two).max() <= 1e-12
