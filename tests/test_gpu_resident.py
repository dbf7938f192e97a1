"""The converged vector stays on the device (the reference reduces its vector
where Davidson left it: OccupationDensity, chemistry/tpb/occupation.h:10-95;
DiagonalReducedDensityMatrix, chemistry/tpb/rdmat.h:10-58; Correlation,
chemistry/tpb/correlation.h:194-444).

A solve run without a host vector leaves its result resident; the density,
alpha weights, RDMs and adjoint computed from the device address must equal
the same reductions of the host copy, and the vector must be the one the
host path returns. Tolerances: 1e-13 (the same kernels on the same data in
a fixed summation order, which agree bit for bit in practice; the tolerance
is a margin)."""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu


def _prob():
    return synth.random_problem(14, 4, 4, 90, 70, seed=21)


def test_resident_vector_equals_host_vector():
    prob = _prob()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        i_h, W = ctx.davidson(max_it=6, max_nb=10, eps=1e-9)
        i_d, none = ctx.davidson(max_it=6, max_nb=10, eps=1e-9, to_host=False)
        assert none is None
        assert i_d.energy == i_h.energy
        Wd = ctx.get_wavefunction(0)
    assert np.array_equal(W, Wd)


def test_reductions_on_resident_vector_match_host_path():
    prob = _prob()
    port = Port()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W = ctx.davidson(max_it=6, max_nb=10, eps=1e-9)
        ptr = ctx.wavefunction_device(0)
        one_d, two_d = ctx.rdm_device(ptr)
        one_h, two_h = ctx.rdm(W)
        assert np.abs(one_d - one_h).max() < 1e-13
        assert np.abs(two_d - two_h).max() < 1e-13
        dens_d = ctx.occupation_device(ptr)
        assert np.abs(dens_d - ctx.occupation(W)).max() < 1e-13
        wa_d = ctx.alpha_weights_device(ptr)
        assert np.abs(wa_d - ctx.alpha_weights(W)).max() < 1e-13
        gh_d, ge_d = ctx.energy_backward_device(ptr)
        gh_h, ge_h = ctx.energy_backward(W)
        assert np.abs(gh_d - gh_h).max() < 1e-12
        assert np.abs(ge_d - ge_h).max() < 1e-12
    # and against the oracle's reductions of the same vector
    one_r, two_r = port.rdm(prob, W)
    assert np.abs(one_d - one_r).max() < 1e-8
    assert np.abs(two_d - two_r).max() < 1e-8
    assert np.abs(dens_d - port.occupation(prob, W)).max() < 1e-12


def test_resident_roots():
    prob = _prob()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        _, E, _, W = ctx.davidson_roots(2, max_it=10, max_nb=10, eps=1e-9)
        _, E2, _, none = ctx.davidson_roots(2, max_it=10, max_nb=10, eps=1e-9, to_host=False)
        assert none is None
        assert np.array_equal(E, E2)
        for r in range(2):
            assert np.array_equal(ctx.get_wavefunction(r), W[r])
        with pytest.raises(sbdx.SbdxError) as e:
            ctx.wavefunction_device(2)
        assert e.value.code == 1


def test_no_solve_no_resident_vector():
    prob = _prob()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        with pytest.raises(sbdx.SbdxError) as e:
            ctx.wavefunction_device(0)
        assert e.value.code == 3
        ctx.davidson(max_it=2, max_nb=6, eps=1e-6, to_host=False)
        ctx.wavefunction_device(0)
        ctx.set_strings(prob.alpha, prob.beta)  # new strings drop it
        with pytest.raises(sbdx.SbdxError):
            ctx.wavefunction_device(0)
