"""Wavefunction files interoperate with the reference's restart format.

The reference writes and reads restart files with SaveWavefunction /
LoadWavefunction (chemistry/tpb/restart.h:20-67, 414-657): three size_t words
(alpha count, beta count, words per string), the strings in bit_length-bit
words, then W alpha-major. The drop-in header (sbd/sbd.h) must read files the
reference wrote and write files the reference reads, giving the same vector
on a new basis (strings missing from the file get zero, the result is
normalised). Runs on the CPU: the compiled reference from oracle/_ref and the
header through the small helper tests/cpp/restart_io.cc.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import Ref
from sbdx import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HELPER_SRC = os.path.join(ROOT, "tests", "cpp", "restart_io.cc")

pytestmark = pytest.mark.skipif(not Ref.available(), reason="reference checker oracle/_ref not built")


@pytest.fixture(scope="module")
def helper(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("restart") / "restart_io")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "sbd-ykt_b200", "cpp", "include"),
           "-I" + os.path.join(ROOT, "include"), "-o", out, HELPER_SRC]
    subprocess.run(cmd, check=True)
    return out


def write_basis(path, L, bl, alpha, beta):
    with open(path, "w") as f:
        f.write(f"{L} {bl} {len(alpha)} {len(beta)}\n")
        f.write("\n".join(str(int(x)) for x in list(alpha) + list(beta)) + "\n")


def run_helper(helper, *args):
    return subprocess.run([helper, *[str(a) for a in args]], capture_output=True, text=True, timeout=120)


def bases(seed=5):
    """A saved basis and a new one that shares part of it, in another order."""
    L = 24
    p1 = synth.random_problem(L, 5, 4, 60, 45, seed=seed)
    p2 = synth.random_problem(L, 5, 4, 70, 50, seed=seed + 1)
    rng = np.random.default_rng(seed)
    a_new = np.unique(np.concatenate([rng.choice(p1.alpha, 40, replace=False), p2.alpha[:30]]))
    b_new = np.unique(np.concatenate([rng.choice(p1.beta, 30, replace=False), p2.beta[:25]]))
    return L, p1.alpha, p1.beta, a_new, b_new


@pytest.mark.parametrize("bl", [20, 64])
def test_reference_written_file_loads(tmp_path, helper, bl):
    L, a0, b0, a1, b1 = bases()
    W0 = np.random.default_rng(1).standard_normal(len(a0) * len(b0))
    ref = Ref()
    stem = str(tmp_path / "wf")
    ref.save_wavefunction(stem, a0, b0, L, W0, bit_length=bl)
    assert os.path.exists(stem + "000000")
    W_ref = ref.load_wavefunction(stem, a1, b1, L, bit_length=bl)
    basis = tmp_path / "basis.txt"
    write_basis(basis, L, bl, a1, b1)
    out = tmp_path / "w.bin"
    r = run_helper(helper, "load", stem, basis, out)
    assert r.returncode == 0, r.stderr
    W = np.fromfile(out, dtype=np.float64)
    assert W.shape == W_ref.shape
    assert np.abs(W - W_ref).max() < 1e-14
    assert abs(np.linalg.norm(W) - 1.0) < 1e-13


def test_header_written_file_loads_in_reference(tmp_path, helper):
    L, a0, b0, a1, b1 = bases(seed=9)
    bl = 20
    W0 = np.random.default_rng(2).standard_normal(len(a0) * len(b0))
    basis0 = tmp_path / "basis0.txt"
    write_basis(basis0, L, bl, a0, b0)
    vin = tmp_path / "w0.bin"
    W0.tofile(vin)
    stem = str(tmp_path / "ours")
    r = run_helper(helper, "save", stem, basis0, vin)
    assert r.returncode == 0, r.stderr
    ref = Ref()
    # same bytes as the reference's own writer
    ref.save_wavefunction(str(tmp_path / "theirs"), a0, b0, L, W0, bit_length=bl)
    assert open(stem + "000000", "rb").read() == open(str(tmp_path / "theirs") + "000000", "rb").read()
    W_ref = ref.load_wavefunction(stem, a1, b1, L, bit_length=bl)
    basis1 = tmp_path / "basis1.txt"
    write_basis(basis1, L, bl, a1, b1)
    out = tmp_path / "w1.bin"
    r = run_helper(helper, "load", stem, basis1, out)
    assert r.returncode == 0, r.stderr
    assert np.abs(np.fromfile(out, dtype=np.float64) - W_ref).max() < 1e-14


def test_truncated_file_is_rejected(tmp_path, helper):
    L, a0, b0, a1, b1 = bases(seed=13)
    ref = Ref()
    stem = str(tmp_path / "wf")
    ref.save_wavefunction(stem, a0, b0, L, np.ones(len(a0) * len(b0)), bit_length=20)
    data = open(stem + "000000", "rb").read()
    open(stem + "000000", "wb").write(data[:-8])
    basis = tmp_path / "basis.txt"
    write_basis(basis, L, 20, a1, b1)
    r = run_helper(helper, "load", stem, basis, tmp_path / "w.bin")
    assert r.returncode == 1
    assert "does not match the file size" in r.stderr
    open(stem + "000000", "wb").write(data[:10])
    r = run_helper(helper, "load", stem, basis, tmp_path / "w.bin")
    assert r.returncode == 1
    assert "LoadWavefunction" in r.stderr
