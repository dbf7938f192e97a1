"""The blocked same-spin kernel (launch codes 31/32/34/38) against the oracle.

The kernel gives a CTA four bra strings that are neighbours in bit-reversed
string order and walks the union of their double-excitation ket lists once
(each ket row strip loaded once, applied to the four strings with their
signed values); the singles and the diagonal stay per string. It computes the
same-spin terms of the reference mult (chemistry/tpb/mult.h:453-552) in
another summation order, so the FP64 sigma must match the oracle's within
1e-12 relative to max |value| and the FP32-storage sigma within 2e-6, for
every column width, on problems whose blocks are split into several work
items (small samples: the split cap is 64 union entries), on the edge shapes,
on row ranges of the alpha strings (shards) and in the pipelined host-buffer
product, whose chunks build blocks over their own rows.
"""
import numpy as np
import pytest
import torch

import sbdx
from sbdx import shard, synth
from oracle import Port

pytestmark = pytest.mark.gpu

CODES = [31, 32, 34, 38]
PROBLEMS = [
    (10, 3, 2, 40, 30, 7),      # unequal electron counts
    (12, 4, 4, 121, 93, 11),    # string counts not multiples of 4 or 8
    (16, 3, 5, 60, 200, 13),
    (24, 5, 5, 150, 150, 17),
    (40, 6, 6, 120, 140, 19),
    (12, 3, 4, 1, 60, 51),      # one alpha string: a block of one
    (12, 4, 3, 70, 1, 52),      # one beta string
    (9, 3, 9, 40, 1, 55),       # full beta spin: no beta excitations
    (64, 6, 5, 121, 93, 58),    # 64 orbitals
]
TOL64, TOL32 = 1e-12, 2e-6


@pytest.fixture(scope="module")
def port():
    return Port()


def _prob(spec):
    L, na_el, nb_el, Na, Nb, seed = spec
    return synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _sigma32(ctx, C):
    dC = torch.tensor(C, dtype=torch.float32, device="cuda")
    dS = torch.empty_like(dC)
    ctx.sigma_device(sbdx.SBDX_FP32, dC.data_ptr(), dS.data_ptr())
    torch.cuda.synchronize()
    return dS.double().cpu().numpy()


@pytest.mark.parametrize("spec", PROBLEMS)
@pytest.mark.parametrize("code", CODES)
def test_blocked_sigma_matches_oracle(spec, code, port):
    prob = _prob(spec)
    C = np.random.default_rng(3).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    ref32 = port.sigma(prob, C.astype(np.float32).astype(np.float64))
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_tuning(code, 71)
        S = ctx.sigma(C)
        assert _rel(S, ref) <= TOL64
        S2 = ctx.sigma(C)
        assert np.array_equal(S, S2)  # fixed summation order: repeatable bit for bit
        assert _rel(_sigma32(ctx, C), ref32) <= TOL32


SKEWED = [("cfg4", 0.25), ("cfg1", 1.0)]


@pytest.mark.parametrize("name,scale", SKEWED)
@pytest.mark.parametrize("code", [32, 34, 38])
def test_blocked_sigma_split_blocks(name, scale, code, port):
    """Near-Aufbau strings of these samples connect to many more strings
    than the mean, so their blocks are split into several work items whose
    partial rows are summed by the fix-up kernel."""
    prob = synth.config(name, scale)
    C = np.random.default_rng(4).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_tuning(code, 71)
        assert _rel(ctx.sigma(C), ref) <= TOL64
        ctx.set_tuning(24, 71)  # the one-string-per-CTA kernel on the same problem
        assert _rel(ctx.sigma(C), ref) <= TOL64


@pytest.mark.parametrize("spec", [PROBLEMS[1], PROBLEMS[4]])
@pytest.mark.parametrize("world", [2, 3])
def test_blocked_row_ranges(spec, world, port):
    prob = _prob(spec)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_tuning(34, 71)
        ctx.build_connectivity()
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        bounds = shard.partition(shard.row_work(ctx), world)
        g = torch.Generator(device="cuda").manual_seed(5)
        C = torch.randn(prob.D, dtype=torch.float64, device="cuda", generator=g)
        S_port = port.sigma(prob, C.cpu().numpy())
        for prec, dt, tol in ((sbdx.SBDX_FP64, torch.float64, TOL64), (sbdx.SBDX_FP32, torch.float32, TOL32)):
            X = C.to(dt)
            S_full = torch.empty_like(X)
            ctx.sigma_device(prec, X.data_ptr(), S_full.data_ptr())
            S_rows = torch.full_like(X, float("nan"))
            for a0, a1 in bounds:
                if a1 > a0:
                    ctx.sigma_rows_device(prec, X.data_ptr(), S_rows[a0 * prob.nb:a1 * prob.nb].data_ptr(), a0, a1)
            torch.cuda.synchronize()
            assert _rel(S_rows.double().cpu().numpy(), S_full.double().cpu().numpy()) < tol
            if prec == sbdx.SBDX_FP64:
                assert _rel(S_rows.cpu().numpy(), S_port) < TOL64


@pytest.mark.parametrize("spec", [PROBLEMS[1], PROBLEMS[3], PROBLEMS[4]])
def test_blocked_pipelined_host_sigma(spec, port):
    prob = _prob(spec)
    C = np.random.default_rng(6).standard_normal(prob.D)
    ref = port.sigma(prob, C)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.set_tuning(34, 71)
        for chunks in (2, 3, 5, 8, 1, 0):
            ctx.set_io_chunks(chunks)
            assert _rel(ctx.sigma(C), ref) <= TOL64, chunks
