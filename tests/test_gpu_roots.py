"""Several lowest roots (sbdx_davidson_roots), FP64 block Davidson and the
mixed-precision solver, against a dense diagonalisation of H whose columns
are the oracle's sigma of unit vectors.

Tolerances: FP64 energies within 1e-9 Ha of the dense eigenvalues, mixed
within 1e-8 Ha; residual norms below eps; Ritz vectors orthonormal to 1e-10
and each within 1e-6 (|<W_r|v_r>| >= 1 - 1e-6) of the dense eigenvector when
that eigenvalue is separated from its neighbours by more than 1e-4 Ha.
"""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

SPECS = [(10, 3, 2, 40, 30, 7), (12, 4, 4, 50, 44, 11), (14, 3, 4, 36, 60, 23)]
_DENSE = {}


def dense(spec, port):
    if spec not in _DENSE:
        L, na_el, nb_el, Na, Nb, seed = spec
        prob = synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)
        D = prob.D
        H = np.zeros((D, D))
        e = np.zeros(D)
        for i in range(D):
            e[i] = 1.0
            H[:, i] = port.sigma(prob, e)
            e[i] = 0.0
        assert np.abs(H - H.T).max() < 1e-10
        w, v = np.linalg.eigh(0.5 * (H + H.T))
        _DENSE[spec] = (prob, w, v)
    return _DENSE[spec]


@pytest.mark.parametrize("spec", SPECS)
@pytest.mark.parametrize("precision,tol", [(sbdx.SBDX_FP64, 1e-9), (sbdx.SBDX_FP32, 1e-8)])
@pytest.mark.parametrize("nroots", [1, 2, 3])
def test_lowest_roots_match_dense(spec, precision, tol, nroots):
    port = Port()
    prob, w, v = dense(spec, port)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, E, res, W = ctx.davidson_roots(nroots, max_it=40, max_nb=12, eps=1e-8, precision=precision)
    assert info.converged == 1
    assert np.all(res < 1e-8)
    assert np.abs(E - w[:nroots]).max() < tol, (E, w[:nroots])
    G = W @ W.T
    assert np.abs(G - np.eye(nroots)).max() < 1e-10
    for r in range(nroots):
        gap = min([abs(w[r] - w[q]) for q in range(len(w)) if q != r])
        if gap > 1e-4:
            assert abs(abs(W[r] @ v[:, r]) - 1.0) < 1e-6


def test_one_root_fp64_block_matches_reference_form():
    """The block solver with one root reaches the energy of the reference
    algorithm (sbdx_davidson, FP64) on the same problem."""
    prob = synth.random_problem(16, 4, 4, 150, 120, seed=31)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        i64, _ = ctx.davidson(max_it=20, max_nb=12, eps=1e-9)
        info, E, res, W = ctx.davidson_roots(1, max_it=20, max_nb=12, eps=1e-9)
    assert info.converged == 1 and i64.converged == 1
    assert abs(E[0] - i64.energy) < 1e-9


def test_roots_argument_errors():
    prob = synth.random_problem(10, 3, 2, 20, 20, seed=3)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        for bad in (0, 5):
            with pytest.raises(sbdx.SbdxError) as e:
                ctx.davidson_roots(bad)
            assert e.value.code == 1
