"""The host-buffer product (sbdx_sigma, the drop-in for mult,
chemistry/tpb/mult.h:376-632) with its copies overlapped with the kernels:
chunks of alpha rows copied in on a second stream, the phase split and the
beta same-spin product per arrived chunk, the alpha-beta product of all
rows, then per chunk the alpha same-spin work items of its rows (added to
the alpha-beta result), the combine and the copy out.

Every chunking must give the oracle's sigma within 1e-12 relative to
max |value| (the FP64 sigma tolerance) and the device-buffer product within
the same bound (the chunks' work items split long rows differently, so the
sums may be grouped differently). Chunk counts from 2 to more than the rows
allow (capped at 8 rows per chunk), row counts that are not multiples of
8, skewed samples whose long rows are split into several work items, a
change of the chunk count between calls, page-locked and pageable host
buffers, and the automatic chunking of a 16 M-determinant problem."""
import numpy as np
import pytest
import torch

import sbdx
from sbdx import synth
from oracle import Port

pytestmark = pytest.mark.gpu

PROBLEMS = [
    (12, 4, 4, 120, 90, 11),
    (16, 3, 5, 60, 200, 13),
    (24, 5, 5, 150, 150, 17),
    (40, 6, 6, 123, 141, 19),  # row counts not multiples of 8
]
TOL = 1e-12


@pytest.fixture(scope="module")
def port():
    return Port()


def _prob(spec):
    L, na_el, nb_el, Na, Nb, seed = spec
    return synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)


def _close(a, b):
    return np.abs(a - b).max() <= TOL * np.abs(b).max()


@pytest.mark.parametrize("spec", PROBLEMS)
def test_chunked_host_sigma_matches_oracle(spec, port):
    prob = _prob(spec)
    C = np.random.default_rng(3).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        for chunks in (2, 3, 5, 8, 64, 1, 0):
            ctx.set_io_chunks(chunks)
            S = ctx.sigma(C)
            assert _close(S, ref), chunks
            S2 = ctx.sigma(C)  # the chunks' work items are reused
            assert _close(S2, ref), chunks


def test_chunked_host_sigma_skewed_split_rows(port):
    """A sample whose near-Aufbau strings connect to many more strings than
    the mean, so that their rows are split into several work items within a
    chunk (as in the parity tests' skewed workloads)."""
    prob = synth.random_problem(18, 4, 4, 700, 64, seed=23)
    C = np.random.default_rng(4).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        for chunks in (2, 7):
            ctx.set_io_chunks(chunks)
            assert _close(ctx.sigma(C), ref), chunks


def test_chunked_host_sigma_pinned_buffers_match_device_product():
    prob = synth.random_problem(24, 5, 5, 400, 380, seed=29)
    gen = torch.Generator().manual_seed(7)
    C = torch.randn(prob.D, dtype=torch.float64, generator=gen)
    hC = C.pin_memory()
    hS = torch.empty_like(hC).pin_memory()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        dC = C.cuda()
        dS = torch.empty_like(dC)
        ctx.sigma_device(sbdx.SBDX_FP64, dC.data_ptr(), dS.data_ptr())
        torch.cuda.synchronize()
        want = dS.cpu().numpy()
        for chunks in (4, 6):
            ctx.set_io_chunks(chunks)
            hS.zero_()
            ctx.sigma_host_ptr(hC.data_ptr(), hS.data_ptr())
            assert _close(hS.numpy(), want), chunks


def test_automatic_chunking_large_problem_matches_device_product():
    """4096 x 4096 strings (16.8 M determinants): the automatic mode runs
    the pipeline with two chunks; the result must equal the device-buffer
    product within the FP64 tolerance."""
    prob = synth.config("cfg2", 0.512)
    assert prob.D >= 16 << 20
    gen = torch.Generator().manual_seed(11)
    C = torch.randn(prob.D, dtype=torch.float64, generator=gen)
    hC = C.pin_memory()
    hS = torch.empty_like(hC).pin_memory()
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        dC = C.cuda()
        dS = torch.empty_like(dC)
        ctx.sigma_device(sbdx.SBDX_FP64, dC.data_ptr(), dS.data_ptr())
        torch.cuda.synchronize()
        want = dS.cpu().numpy()
        del dC, dS
        ctx.sigma_host_ptr(hC.data_ptr(), hS.data_ptr())
        assert _close(hS.numpy(), want)


def test_io_chunks_argument_checked():
    prob = _prob(PROBLEMS[0])
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        with pytest.raises(sbdx.SbdxError):
            ctx.set_io_chunks(-1)
