"""Error of the mixed-precision solve's RDMs against the FP64 oracle.

The mixed solver (FP32-stored corrections and FP32-storage sigmas, FP64
anchors refreshed by exact FP64 sigmas, FP64 Rayleigh-Ritz and residuals)
must give the same state as the plain FP64 form: its energies within 1e-9 Ha
and the 1-/2-RDMs of its vectors within 1e-8 max-abs of the oracle's RDMs
(oracle/sbd_oracle.c, the restatement of Correlation,
chemistry/tpb/correlation.h:194-444) of the FP64 vector. Both solves run to
a 1e-10 residual so that the vectors themselves agree well below the RDM
tolerance. Workloads: the CPU-runnable synthetic workload (L = 24, 5+5
electrons, 400 x 400 strings) and the differentiation workload scaled to
500 x 500 strings (L = 32, 6+6 electrons), one and two roots.
"""
import numpy as np
import pytest

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

RDM_TOL = 1e-8
E_TOL = 1e-9


@pytest.fixture(scope="module")
def port():
    return Port()


@pytest.mark.parametrize("name, scale", [("cfg1", 1.0), ("cfg4", 0.25)])
@pytest.mark.parametrize("defect_every", [0, 4])
def test_mixed_single_root_rdm(name, scale, defect_every, port):
    prob = synth.config(name, scale)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        i64, _ = ctx.davidson(max_it=100, max_nb=12, eps=1e-10, to_host=False)
        W64 = ctx.get_wavefunction(0)
        i32, _ = ctx.davidson(max_it=100, max_nb=12, eps=1e-10, precision=sbdx.SBDX_FP32,
                              defect_every=defect_every, to_host=False)
        assert i32.converged == 1 and i64.converged == 1
        one32, two32 = ctx.rdm_device(ctx.wavefunction_device(0))
    one_r, two_r = port.rdm(prob, W64)
    assert abs(i32.energy - i64.energy) < E_TOL
    assert np.abs(one32 - one_r).max() < RDM_TOL
    assert np.abs(two32 - two_r).max() < RDM_TOL
    # the RDM energy identity of the mixed state reproduces the FP64 energy
    assert abs(port.rdm_energy(prob, one32, two32) - i64.energy) < E_TOL


def test_mixed_two_roots_rdm(port):
    prob = synth.config("cfg1")
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        f64, E64, _, W64 = ctx.davidson_roots(2, max_it=100, max_nb=12, eps=1e-10)
        f32, E32, _, _ = ctx.davidson_roots(2, max_it=100, max_nb=12, eps=1e-10, precision=sbdx.SBDX_FP32,
                                            defect_every=4, to_host=False)
        assert f64.converged == 1 and f32.converged == 1
        rdms = [ctx.rdm_device(ctx.wavefunction_device(r)) for r in range(2)]
    assert np.abs(E32 - E64).max() < E_TOL
    for r in range(2):
        one_r, two_r = port.rdm(prob, W64[r])
        assert np.abs(rdms[r][0] - one_r).max() < RDM_TOL
        assert np.abs(rdms[r][1] - two_r).max() < RDM_TOL
