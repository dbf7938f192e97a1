"""The subspace projection of the Davidson solvers on the FP64 tensor pipe
(sbdx_project_device): P[i][r] = <V_i, X_r> for m vectors V and up to 8
vectors X. The reference evaluates these dots one pair at a time
(InnerProduct, framework/dm_vector.h:179-243; called from
chemistry/tpb/davidson.h:756-797 and 865-873).

Checked against a torch FP64 matrix product of the same vectors (FP32
vectors widened to FP64 first, as the kernel does): relative error at most
1e-13 of sum_d |V_i[d] X_r[d]|, the bound of an FP64 sum of D products in any
order. Shapes cover a few dots with one vector (the CUDA-core kernel), one
row tile and several, more than 64 rows (further grid
rows), every column count, lengths that are not a multiple of the 32-element
chunk or of 4 (the element-wise path), strides above D and unaligned starts;
a repeated call must give identical bits (fixed-order reduction)."""
import numpy as np
import pytest
import torch

import sbdx

pytestmark = pytest.mark.gpu


def _ctx():
    return sbdx.Context(0)


def _check(ctx, prec, m, nx, D, ldv=None, ldx=None, off=0, seed=0):
    dt = torch.float32 if prec == sbdx.SBDX_FP32 else torch.float64
    ldv = D if ldv is None else ldv
    ldx = D if ldx is None else ldx
    g = torch.Generator(device="cuda").manual_seed(seed)
    vbuf = torch.randn(off + max(m, 1) * ldv, generator=g, device="cuda", dtype=torch.float64).to(dt)
    xbuf = torch.randn(off + nx * ldx, generator=g, device="cuda", dtype=torch.float64).to(dt)
    V = vbuf[off:off + m * ldv].view(m, ldv)[:, :D] if m else vbuf[:0]
    X = xbuf[off:off + nx * ldx].view(nx, ldx)[:, :D]
    P = torch.empty(max(m * nx, 1), device="cuda", dtype=torch.float64)
    ctx.project_device(prec, vbuf.data_ptr() + off * vbuf.element_size(), ldv, m,
                       xbuf.data_ptr() + off * xbuf.element_size(), ldx, nx, D, P.data_ptr())
    if m == 0:
        return
    got = P[:m * nx].view(m, nx)
    Vd, Xd = V.double(), X.double()
    want = Vd @ Xd.T
    scale = Vd.abs() @ Xd.abs().T
    err = ((got - want).abs() / scale.clamp_min(1e-300)).max().item()
    assert err <= 1e-13, (prec, m, nx, D, err)
    P2 = torch.empty_like(P)
    ctx.project_device(prec, vbuf.data_ptr() + off * vbuf.element_size(), ldv, m,
                       xbuf.data_ptr() + off * xbuf.element_size(), ldx, nx, D, P2.data_ptr())
    assert torch.equal(P, P2)


@pytest.mark.parametrize("prec", [sbdx.SBDX_FP64, sbdx.SBDX_FP32])
@pytest.mark.parametrize("m", [1, 3, 8, 9, 16, 17, 32, 33, 64, 65, 130])
def test_projection_row_counts(prec, m):
    with _ctx() as ctx:
        for nx in (1, 2, 5, 8):
            _check(ctx, prec, m, nx, 4096 + 32 * 7, seed=m * 10 + nx)


@pytest.mark.parametrize("prec", [sbdx.SBDX_FP64, sbdx.SBDX_FP32])
@pytest.mark.parametrize("D", [1, 3, 31, 33, 1000, 4099, 100003, 1 << 20])
def test_projection_lengths(prec, D):
    with _ctx() as ctx:
        _check(ctx, prec, 20, 2, D, seed=D)
        _check(ctx, prec, 2, 1, D, seed=D + 1)


@pytest.mark.parametrize("prec", [sbdx.SBDX_FP64, sbdx.SBDX_FP32])
def test_projection_strides_and_unaligned_starts(prec):
    with _ctx() as ctx:
        _check(ctx, prec, 12, 3, 5000, ldv=5003, ldx=5001)
        _check(ctx, prec, 12, 3, 5000, off=1)
        _check(ctx, prec, 40, 8, 4096, ldv=4100, ldx=4104, off=2)
        _check(ctx, prec, 2, 1, 4096, off=1)  # a few dots with one vector: the CUDA-core kernel
        _check(ctx, prec, 3, 1, 4096, ldv=4098)


def test_projection_empty_and_bad_arguments():
    with _ctx() as ctx:
        _check(ctx, sbdx.SBDX_FP64, 0, 1, 100)
        X = torch.zeros(100, device="cuda", dtype=torch.float64)
        P = torch.zeros(16, device="cuda", dtype=torch.float64)
        with pytest.raises(sbdx.SbdxError):
            ctx.project_device(sbdx.SBDX_FP64, X.data_ptr(), 100, 1, X.data_ptr(), 100, 9, 100, P.data_ptr())
        with pytest.raises(sbdx.SbdxError):
            ctx.project_device(sbdx.SBDX_FP64, X.data_ptr(), 50, 2, X.data_ptr(), 100, 1, 100, P.data_ptr())


def test_projection_large_vectors_match_numpy_dots():
    """400 M-element scale is not needed for the arithmetic; 2^25 elements
    (FP32, 20 vectors: 2.7 GB) checks the grid-stride loop over many chunks
    per warp against FP64 dots on the host of a few sampled pairs."""
    D, m = 1 << 25, 20
    with _ctx() as ctx:
        g = torch.Generator(device="cuda").manual_seed(5)
        V = torch.randn(m, D, generator=g, device="cuda", dtype=torch.float32)
        X = torch.randn(2, D, generator=g, device="cuda", dtype=torch.float32)
        P = torch.empty(m * 2, device="cuda", dtype=torch.float64)
        ctx.project_device(sbdx.SBDX_FP32, V.data_ptr(), D, m, X.data_ptr(), D, 2, D, P.data_ptr())
        got = P.view(m, 2).cpu().numpy()
        Xh = X.double().cpu().numpy()
        for i in (0, 7, 19):
            vi = V[i].double().cpu().numpy()
            for r in range(2):
                want = float(np.dot(vi, Xh[r]))
                scale = float(np.dot(np.abs(vi), np.abs(Xh[r])))
                assert abs(got[i, r] - want) <= 1e-13 * scale
