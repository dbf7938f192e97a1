"""Energy adjoint (sbdx_energy_backward) and its torch.autograd binding.

dE/d(integral entry) from the backward kernel must match central finite
differences of the forward solve (step 1e-5, 1e-6 relative agreement) on
seeded entries, and the RDM contraction of the oracle (the reference's
Correlation restated) to 1e-10.
"""
import numpy as np
import pytest
import torch

import sbdx
from sbdx import autograd as sag
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu


def rdm_gradient(prob, one, two):
    """dE/dh_pair and dE/d(class) from RDMs, restating the sample's energy
    identity (main.cc:166-216) differentiated entry by entry."""
    L = prob.L
    g1 = (one[: L * L] + one[L * L:]).reshape(L, L).T  # g1[p, q] = gamma[p + L q]
    dh = g1 + g1.T - np.diag(np.diag(g1))
    G = two.reshape(4, L, L, L, L).sum(0)  # G[l, k, j, i] = sum_s two[s][i + L j + L^2 k + L^3 l]
    deri = np.zeros(synth.neri(L))
    for io in range(L):
        for jo in range(L):
            for ia in range(L):
                for ja in range(L):
                    deri[synth.eri_index(io, ia, jo, ja)] += 0.5 * G[ja, ia, jo, io]
    return dh, deri


def test_backward_matches_rdm_contraction():
    prob = synth.random_problem(10, 3, 3, 60, 50, seed=17, K=12)
    port = Port()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W = ctx.davidson(max_it=20, max_nb=12, eps=1e-11)
        dh, deri = ctx.energy_backward(W)
    one, two = port.rdm(prob, W)
    rdh, rderi = rdm_gradient(prob, one, two)
    assert np.abs(dh.reshape(prob.L, prob.L) - rdh).max() < 1e-10
    assert np.abs(deri - rderi).max() < 1e-10


def test_autograd_matches_central_differences():
    prob = synth.random_problem(16, 4, 4, 150, 150, seed=23, K=24)
    L = prob.L
    h_tri = torch.tensor(sag.tril_pack(prob.h.reshape(L, L)), requires_grad=True)
    eri = torch.tensor(prob.eri, requires_grad=True)
    with sbdx.Context(0) as ctx:
        ctx.set_strings(prob.alpha, prob.beta)
        E = sag.energy(ctx, h_tri, eri, L, prob.I0)
        E.backward()
        gh, ge = h_tri.grad.numpy().copy(), eri.grad.numpy().copy()
        rng = np.random.default_rng(5)
        picks = [("h", int(i)) for i in rng.choice(len(h_tri), 32, replace=False)]
        nz = np.flatnonzero(np.abs(prob.eri) > 1e-3)
        picks += [("e", int(i)) for i in rng.choice(nz, 32, replace=False)]  # 64 entries in all
        step = 1e-5
        for kind, i in picks:
            vals = []
            for sgn in (+1, -1):
                ht = h_tri.detach().clone()
                et = eri.detach().clone()
                (ht if kind == "h" else et)[i] += sgn * step
                vals.append(float(sag.energy(ctx, ht, et, L, prob.I0)))
            fd = (vals[0] - vals[1]) / (2 * step)
            an = gh[i] if kind == "h" else ge[i]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (kind, i, fd, an)


def test_products_after_backward_rebuild_full_connectivity():
    """The backward pass rebuilds only the excitation lists; a later sigma,
    RDM and solve on the same context must rebuild what they need and agree
    with the oracle (FP64 sigma 1e-12 relative, energy 1e-9 Ha)."""
    prob = synth.random_problem(14, 4, 4, 90, 110, seed=29, K=12)
    port = Port()
    C = np.random.default_rng(7).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W = ctx.davidson(max_it=20, max_nb=12, eps=1e-10)
        ctx.energy_backward(W)
        sl, dl, idx = ctx.connectivity(0)  # the lists are there
        rsl, rdl, ridx = port.connectivity(prob.alpha)
        assert np.array_equal(sl, rsl) and np.array_equal(dl, rdl) and np.array_equal(idx, ridx)
        S = ctx.sigma(C)
        assert np.abs(S - ref).max() <= 1e-12 * np.abs(ref).max()
        one, two = ctx.rdm(W)
        r1, r2 = port.rdm(prob, W)
        assert np.abs(one - r1).max() < 1e-8 and np.abs(two - r2).max() < 1e-8
        info2, _ = ctx.davidson(max_it=20, max_nb=12, eps=1e-10)
        assert abs(info2.energy - info.energy) < 1e-9
