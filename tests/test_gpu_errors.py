"""Error behaviour of the C-ABI: invalid host inputs return error codes with a
message and leave the context usable; nothing reaches a kernel."""
import numpy as np
import pytest

import sbdx
from sbdx import synth

pytestmark = pytest.mark.gpu


def codes(fn):
    with pytest.raises(sbdx.SbdxError) as e:
        fn()
    return e.value.code


def test_invalid_inputs_are_reported():
    prob = synth.random_problem(10, 3, 3, 30, 30, seed=2)
    with sbdx.Context(0) as ctx:
        assert codes(lambda: ctx.sigma(np.zeros(4))) == 3          # before set_strings
        bad = prob.eri.copy()
        bad[7] = np.nan
        assert codes(lambda: ctx.set_integrals(prob.L, prob.I0, prob.h, bad)) == 5
        assert codes(lambda: ctx.set_integrals(prob.L, prob.I0, prob.h, prob.eri[:-1])) == 1
        assert codes(lambda: ctx.set_integrals(65, prob.I0, np.zeros(65 * 65), np.zeros(synth.neri(65)))) == 1
        a = prob.alpha.copy()
        a[3] = a[3] | (1 << 9) | (1 << 8)
        assert codes(lambda: ctx.set_strings(a, prob.beta)) == 1   # unequal electron count
        ctx.load(prob)
        assert codes(lambda: ctx.davidson(max_nb=0)) == 1
        hi = prob.alpha.copy()
        hi[0] = (hi[0] & ~np.uint64(1)) | np.uint64(1 << 12)       # orbital beyond norb = 10
        ctx.set_strings(hi, prob.beta)
        assert codes(lambda: ctx.diag_terms()) == 1
        ctx.set_strings(prob.alpha, prob.beta)                     # still usable afterwards
        S = ctx.sigma(np.ones(prob.D))
        assert np.isfinite(S).all()


def test_davidson_time_guard_stops_early():
    prob = synth.random_problem(14, 4, 4, 120, 120, seed=4)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W = ctx.davidson(max_it=50, max_nb=12, eps=1e-14, max_time=0.0)
        assert info.converged == 0 and info.n_sigma <= 3
        assert abs(np.linalg.norm(W) - 1) < 1e-12
