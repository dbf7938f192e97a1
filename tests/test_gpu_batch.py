"""Batches of subspaces (sbdx_batch_*): every subspace of a batch solved
concurrently must give what a separate context gives for it.

Tolerances: FP64 energies within 1e-9 Ha of sbdx_davidson_roots on a separate
context, mixed precision within 1e-8 Ha; exact residuals below eps; the
returned Ritz vectors have unit norm and Rayleigh quotient equal to the
energy (1e-9 Ha, through the oracle's sigma)."""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu


def subspaces(L=14, n=4, sizes=((30, 40), (90, 60), (12, 200), (150, 140), (8, 9), (60, 61)), seed=41):
    I0, h, eri = synth.make_integrals(L, 8, seed)
    subs = []
    for k, (na, nb) in enumerate(sizes):
        a = synth.sample_strings(L, n, na, seed + 10 + 2 * k)
        b = synth.sample_strings(L, n, nb, seed + 11 + 2 * k)
        subs.append(synth.Problem(L=L, nelec=2 * n, I0=I0, h=h, eri=eri, alpha=a, beta=b))
    return subs


@pytest.mark.parametrize("precision,tol", [(sbdx.SBDX_FP64, 1e-9), (sbdx.SBDX_FP32, 1e-8)])
@pytest.mark.parametrize("nthreads", [1, 4])
def test_batch_matches_separate_solves(precision, tol, nthreads):
    subs = subspaces()
    nroots = 2
    ref = []
    for p in subs:
        with sbdx.Context(0) as ctx:
            ctx.load(p)
            info, E, res, _ = ctx.davidson_roots(nroots, max_it=40, max_nb=10, eps=1e-9, precision=sbdx.SBDX_FP64)
            assert info.converged == 1
            ref.append(E)
    p0 = subs[0]
    with sbdx.Batch(p0.L, p0.I0, p0.h, p0.eri) as batch:
        for p in subs:
            batch.add(p.alpha, p.beta)
        E, R, infos, sec = batch.solve(nroots=nroots, max_it=40, max_nb=10, eps=1e-9, precision=precision,
                                       nthreads=nthreads)
        assert sec > 0
        for k, p in enumerate(subs):
            assert infos[k].converged == 1
            assert np.all(R[k] < 1e-9)
            assert np.abs(E[k] - ref[k]).max() < tol, (k, E[k], ref[k])
        port = Port()
        for k in (1, 3):
            W = batch.vector(k, 1)
            assert abs(np.linalg.norm(W) - 1.0) < 1e-10
            rq = W @ port.sigma(subs[k], W)
            assert abs(rq - E[k, 1]) < 1e-9


def test_batch_tune_and_errors():
    subs = subspaces(sizes=((40, 50), (20, 25)))
    p0 = subs[0]
    with sbdx.Batch(p0.L, p0.I0, p0.h, p0.eri) as batch:
        with pytest.raises(sbdx.SbdxError):
            batch.solve(nroots=1)  # empty batch
        for p in subs:
            batch.add(p.alpha, p.beta)
        s, a = batch.tune()
        assert s > 0 and a > 0
        with pytest.raises(sbdx.SbdxError) as e:
            batch.solve(nroots=5)
        assert e.value.code == 1
        E, R, infos, _ = batch.solve(nroots=1, eps=1e-8)
        assert all(i.converged == 1 for i in infos)
        with pytest.raises(sbdx.SbdxError):
            batch.vector(0, 1)  # only one root solved
