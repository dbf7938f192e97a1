"""sbdx_diag_terms_noalloc: the diagonal H_II from caller-owned device buffers
with the library's fixed scratch array instead of any device allocation.

The GPU tests call the C-ABI entry point on torch device tensors and compare
with sbdx_diag_terms (the context entry point) on the same problem. Tolerance:
|noalloc - diag_terms| <= 1e-12 * max(1, |diag_terms|) elementwise; both sum the
same terms in the same order, so they normally agree bit for bit.

The file name sorts last so that the first call of the process (the scratch
address look-up) also happens after every other test has used the library.
"""
import ctypes

import numpy as np
import pytest

import sbdx
from sbdx import synth

SCRATCH_DOUBLES = 1 << 19
RTOL = 1e-12


def reference_hii(prob):
    with sbdx.Context(0) as ctx:
        ctx.load(prob)
        return ctx.diag_terms()


def call_noalloc(prob, torch, stream):
    dev = torch.device("cuda", 0)
    h = torch.from_numpy(np.ascontiguousarray(prob.h, dtype=np.float64)).to(dev)
    eri = torch.from_numpy(np.ascontiguousarray(prob.eri, dtype=np.float64)).to(dev)
    a = torch.from_numpy(prob.alpha.view(np.int64)).to(dev)
    b = torch.from_numpy(prob.beta.view(np.int64)).to(dev)
    hii = torch.full((prob.D,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    sbdx.diag_terms_noalloc(prob.L, prob.I0, h.data_ptr(), eri.data_ptr(), a.data_ptr(), prob.na, b.data_ptr(),
                            prob.nb, hii.data_ptr(), stream.cuda_stream)
    return hii, (h, eri, a, b)


def assert_close(got, want):
    err = np.abs(got - want)
    assert np.all(err <= RTOL * np.maximum(1.0, np.abs(want))), float(err.max())


@pytest.mark.gpu
def test_two_calls_in_a_row_match_diag_terms():
    torch = pytest.importorskip("torch")
    small = synth.random_problem(14, 4, 3, 120, 90, seed=11)
    # na + nb + nb*L = 5088 + 8800 * 59 = 524288: exactly the scratch size
    L, n = 58, 7
    I0, h, eri = synth.make_integrals(L, 16, seed=77)
    large = synth.Problem(L=L, nelec=2 * n, I0=I0, h=h, eri=eri, alpha=synth.sample_strings(L, n, 5088, 78),
                          beta=synth.sample_strings(L, n, 8800, 79))
    assert large.na + large.nb * (L + 1) == SCRATCH_DOUBLES
    want_small = reference_hii(small)
    want_large = reference_hii(large)

    stream = torch.cuda.Stream()
    # small, then large (reads scratch words the small call left behind), then
    # small again: every call must write what it reads
    for prob, want in ((small, want_small), (large, want_large), (small, want_small)):
        hii, keep = call_noalloc(prob, torch, stream)
        stream.synchronize()
        assert_close(hii.cpu().numpy(), want)
        del keep


@pytest.mark.gpu
def test_oversize_is_rejected_before_any_launch():
    torch = pytest.importorskip("torch")
    prob = synth.random_problem(10, 3, 3, 30, 30, seed=4)
    dev = torch.device("cuda", 0)
    buf = torch.zeros(64, dtype=torch.float64, device=dev)
    hii = torch.full((16,), 7.0, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    with pytest.raises(sbdx.SbdxError) as e:
        # 1 + 262144 + 262144 * 1 = 524289 doubles of scratch
        sbdx.diag_terms_noalloc(1, prob.I0, p, p, p, 1, p, 262144, hii.data_ptr(), 0)
    assert e.value.code == 1 and "exceeds the fixed scratch" in str(e.value)
    torch.cuda.synchronize()
    assert torch.all(hii == 7.0)  # nothing was launched
    # the library is still usable afterwards
    got, keep = call_noalloc(prob, torch, torch.cuda.current_stream())
    torch.cuda.synchronize()
    assert_close(got.cpu().numpy(), reference_hii(prob))


def test_argument_errors_need_no_gpu():
    """Host-side validation runs before anything touches a pointer or CUDA."""
    lib = sbdx.load_library()
    fn = lib.sbdx_diag_terms_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_double] + [ctypes.c_void_p] * 3 + [ctypes.c_size_t, ctypes.c_void_p,
                                                                           ctypes.c_size_t, ctypes.c_void_p,
                                                                           ctypes.c_void_p, ctypes.c_char_p,
                                                                           ctypes.c_size_t]
    buf = ctypes.create_string_buffer(200)
    fake = 4096  # never dereferenced: every case below fails its argument check
    assert fn(0, 0.0, fake, fake, fake, 4, fake, 4, fake, None, buf, 200) == 1
    assert b"norb" in buf.value
    assert fn(65, 0.0, fake, fake, fake, 4, fake, 4, fake, None, buf, 200) == 1
    assert fn(8, 0.0, None, fake, fake, 4, fake, 4, fake, None, buf, 200) == 1
    assert b"null pointer" in buf.value
    assert fn(8, 0.0, fake, fake, fake, 0, fake, 4, fake, None, buf, 200) == 1
    assert fn(8, 0.0, fake, fake, fake, 65536, fake, 4, fake, None, buf, 200) == 1
    assert fn(64, 0.0, fake, fake, fake, 1000, fake, 8100, fake, None, buf, 200) == 1
    assert b"exceeds the fixed scratch of 524288 doubles" in buf.value
    small = ctypes.create_string_buffer(8)
    assert fn(64, 0.0, fake, fake, fake, 1000, fake, 8100, fake, None, small, 8) == 1
    assert small.value == b"diag_te"  # truncated and NUL-terminated
