"""The device-driven several-root solver (sbdx_set_graph_steps): one CUDA graph
per Davidson iteration, the generalised Rayleigh-Ritz problem solved on the
device, the host reading each iteration's status one iteration later.

It must reach what the host-driven solver reaches: the lowest eigenvalues of
a dense diagonalisation (FP64 within 1e-9 Ha, mixed precision within 1e-8 Ha,
including a refresh every 4 iterations), residuals below eps, orthonormal
Ritz vectors; the same on the legacy stream (no capture, the same kernels);
and a batch with graph steps must match separate solves."""
import numpy as np
import pytest
import torch

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

SPECS = [(10, 3, 2, 40, 30, 7), (12, 4, 4, 50, 44, 11), (14, 3, 4, 36, 60, 23)]
_DENSE = {}


def dense(spec):
    if spec not in _DENSE:
        port = Port()
        prob = synth.random_problem(*spec)
        H = np.zeros((prob.D, prob.D))
        e = np.zeros(prob.D)
        for i in range(prob.D):
            e[i] = 1.0
            H[:, i] = port.sigma(prob, e)
            e[i] = 0.0
        w, v = np.linalg.eigh(0.5 * (H + H.T))
        _DENSE[spec] = (prob, w)
    return _DENSE[spec]


@pytest.mark.parametrize("spec", SPECS)
@pytest.mark.parametrize("precision,tol,every", [(sbdx.SBDX_FP64, 1e-9, 0), (sbdx.SBDX_FP32, 1e-8, 0),
                                                 (sbdx.SBDX_FP32, 1e-8, 4)])
@pytest.mark.parametrize("nroots", [1, 2, 3])
def test_graph_steps_match_dense(spec, precision, tol, every, nroots):
    prob, w = dense(spec)
    stream = torch.cuda.Stream()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_stream(stream.cuda_stream)
        ctx.set_graph_steps(True)
        info, E, res, W = ctx.davidson_roots(nroots, max_it=40, max_nb=12, eps=1e-8, precision=precision,
                                             defect_every=every)
    assert info.converged == 1
    assert np.all(res < 1e-8)
    assert np.abs(E - w[:nroots]).max() < tol, (E, w[:nroots])
    assert np.abs(W @ W.T - np.eye(nroots)).max() < 1e-10


@pytest.mark.parametrize("precision,tol", [(sbdx.SBDX_FP64, 1e-9), (sbdx.SBDX_FP32, 1e-8)])
def test_graph_steps_on_legacy_stream_and_larger_problem(precision, tol):
    prob = synth.random_problem(24, 5, 5, 150, 150, seed=17)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        _, E_ref, _, _ = ctx.davidson_roots(2, max_it=40, max_nb=12, eps=1e-9)
        ctx.set_graph_steps(True)  # legacy stream: the same kernels, no graphs
        info, E, res, _ = ctx.davidson_roots(2, max_it=40, max_nb=12, eps=1e-9, precision=precision)
        assert info.converged == 1 and np.all(res < 1e-9)
        assert np.abs(E - E_ref).max() < tol
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        info, E2, res2, _ = ctx.davidson_roots(2, max_it=40, max_nb=12, eps=1e-9, precision=precision)
        assert info.converged == 1 and np.all(res2 < 1e-9)
        assert np.abs(E2 - E_ref).max() < tol


def test_batch_with_graph_steps_matches_separate_solves():
    L, n = 14, 4
    I0, h, eri = synth.make_integrals(L, 8, 41)
    sizes = ((30, 40), (90, 60), (12, 200), (150, 140), (8, 9), (60, 61))
    subs = []
    for k, (na, nb) in enumerate(sizes):
        a = synth.sample_strings(L, n, na, 51 + 2 * k)
        b = synth.sample_strings(L, n, nb, 52 + 2 * k)
        subs.append(synth.Problem(L=L, nelec=2 * n, I0=I0, h=h, eri=eri, alpha=a, beta=b))
    ref = []
    for p in subs:
        with sbdx.Context(0) as ctx:
            ctx.load(p)
            info, E, _, _ = ctx.davidson_roots(2, max_it=40, max_nb=10, eps=1e-9)
            ref.append(E)
    with sbdx.Batch(L, I0, h, eri) as batch:
        for p in subs:
            batch.add(p.alpha, p.beta)
        batch.set_graph_steps(True)
        for prec, tol in ((sbdx.SBDX_FP64, 1e-9), (sbdx.SBDX_FP32, 1e-8)):
            E, R, infos, _ = batch.solve(nroots=2, max_it=40, max_nb=10, eps=1e-9, precision=prec, nthreads=4)
            assert all(i.converged for i in infos)
            assert np.all(R < 1e-9)
            assert np.abs(E - np.array(ref)).max() < tol
