"""Connectivity of the full-size workloads, bit-exact against the oracle.

The helper lists (GenerateExcitation + MakeSmartHelper, chemistry/tpb/
helper.h:132-197, 367-437: per bra string its singles then its doubles,
ascending ket index) of both spins of the plain FP64 drop-in workload
(8000 x 8000 strings, L = 58) and of the mixed-precision workload
(20000 x 20000 strings) must equal the C restatement's
(oracle/sbd_oracle.c, sbo_connectivity) entry for entry."""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cfg2", "cfg3"])
def test_full_size_connectivity_bit_exact(name):
    prob = synth.config(name)
    port = Port()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        for spin, strings in ((0, prob.alpha), (1, prob.beta)):
            sl, dl, idx = ctx.connectivity(spin)
            rsl, rdl, ridx = port.connectivity(strings)
            assert np.array_equal(sl, rsl)
            assert np.array_equal(dl, rdl)
            assert np.array_equal(idx, ridx)
