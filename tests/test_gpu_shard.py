"""Row-range products and the sharded solve on the GPU (one process).

sbdx_sigma_rows_device evaluates output rows [a0, a1) of S = H C from the
whole C: the blocks of a partition into 2 and 3 shards, computed one after
another on one GPU (no kernel waits on another), must reassemble the whole
product (FP64 within 1e-12 relative, FP32 storage within 2e-6 relative of
the whole FP32 product). The sharded FP64 Davidson (sbdx/shard.py) at world
size 1 over the row-range product must give the single-GPU solver's energy
within 1e-9 Ha. Problems include strings split into several work items (a
skewed sample) and alpha rows that own no single excitation."""
import numpy as np
import pytest
import torch

import sbdx
from sbdx import shard, synth
from oracle import Port

pytestmark = pytest.mark.gpu

PROBLEMS = [
    (14, 4, 4, 90, 70, 21),
    (24, 5, 5, 150, 150, 17),
    (16, 3, 5, 60, 200, 13),
]


def _prob(spec):
    return synth.random_problem(*spec)


@pytest.mark.parametrize("spec", PROBLEMS)
@pytest.mark.parametrize("world", [2, 3])
def test_row_blocks_reassemble_the_product(spec, world):
    prob = _prob(spec)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        bounds = shard.partition(shard.row_work(ctx), world)
        g = torch.Generator(device="cuda").manual_seed(5)
        C = torch.randn(prob.D, dtype=torch.float64, device="cuda", generator=g)
        for prec, dt, tol in ((sbdx.SBDX_FP64, torch.float64, 1e-12), (sbdx.SBDX_FP32, torch.float32, 2e-6)):
            X = C.to(dt)
            S_full = torch.empty_like(X)
            ctx.sigma_device(prec, X.data_ptr(), S_full.data_ptr())
            S_rows = torch.full_like(X, float("nan"))
            for a0, a1 in bounds:
                if a1 > a0:
                    out = S_rows[a0 * prob.nb:a1 * prob.nb]
                    ctx.sigma_rows_device(prec, X.data_ptr(), out.data_ptr(), a0, a1)
            torch.cuda.synchronize()
            ref = S_full.double()
            err = float((S_rows.double() - ref).abs().max() / ref.abs().max())
            assert err < tol, (prec, err)
            if prec == sbdx.SBDX_FP64:  # and the oracle's whole product
                S_port = Port().sigma(prob, C.cpu().numpy())
                assert np.abs(S_rows.cpu().numpy() - S_port).max() / np.abs(S_port).max() < 1e-12


def test_row_range_arguments():
    prob = _prob(PROBLEMS[0])
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        C = torch.zeros(prob.D, dtype=torch.float64, device="cuda")
        S = torch.zeros(prob.D, dtype=torch.float64, device="cuda")
        with pytest.raises(sbdx.SbdxError) as e:
            ctx.sigma_rows_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr(), 4, 20)  # a0 not a multiple of 8
        assert e.value.code == 1
        with pytest.raises(sbdx.SbdxError):
            ctx.sigma_rows_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr(), 8, prob.na + 1)
        with pytest.raises(sbdx.SbdxError):  # output overlapping the input
            ctx.sigma_rows_device(sbdx.SBDX_FP64, C.data_ptr(), C.data_ptr(), 0, 8)
        ctx.sigma_rows_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr(), 8, 8)  # empty range


@pytest.mark.parametrize("spec", PROBLEMS[:2])
def test_sharded_davidson_world_one(spec):
    prob = _prob(spec)
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        info, W_ref = ctx.davidson(max_it=6, max_nb=10, eps=1e-9)
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        comm = shard.Comm()
        bounds = shard.partition(shard.row_work(ctx), 1)
        op = shard.ShardedSigma(ctx, comm, bounds)
        hii = torch.from_numpy(ctx.diag_terms()).cuda()
        W0 = torch.zeros(prob.D, dtype=torch.float64, device="cuda")
        W0[0] = 1.0
        E, W, inf = shard.davidson(op, hii, comm, W0, max_it=6, max_nb=10, eps=1e-9)
    assert abs(E - info.energy) < 1e-9
    assert abs(abs(float(np.dot(W.cpu().numpy(), W_ref))) - 1.0) < 1e-8
