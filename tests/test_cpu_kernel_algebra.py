"""CPU model of the algebra the CUDA kernels use, checked exhaustively against
the reference's interleaved-determinant Slater-Condon rules (the oracle's Hij).

The kernels never build the 2L-bit interleaved determinant. They split every
fermionic sign into a same-spin part, computed once per connectivity entry,
and an opposite-spin part, a parity of (opposite-spin string & mask); the
alpha-beta kernel uses prefix-parity words. This test re-derives H_IJ for
every connected pair of small problems from exactly those pieces.
"""
import numpy as np
import pytest

from oracle import Port
from sbdx import synth


def popc(x):
    return bin(int(x)).count("1")


def rmask(lo, hi):
    return ((1 << hi) - 1) & ~((1 << lo) - 1)


def other_range(spin, x, y):
    return rmask(x, y) if spin == 0 else rmask(x + 1, y + 1)


def prefix_parity(s):
    out, acc = 0, 0
    for p in range(64):
        acc ^= (s >> p) & 1
        out |= acc << p
    return out


def eri(prob, p, q, r, s):
    return prob.eri[synth.eri_index(p, q, r, s)]


def entry(prob, spin, sr, sk):
    """Same-spin part of <bra|H|ket> (the connectivity builder's make_entry)."""
    L = prob.L
    h = prob.h.reshape(L, L)
    hole, part = sk & ~sr, sr & ~sk
    if popc(hole) == 1:
        i, a = hole.bit_length() - 1, part.bit_length() - 1
        lo, hi = min(i, a), max(i, a)
        neg = popc(sk & rmask(lo + 1, hi)) & 1
        v = h[a, i] + sum(eri(prob, a, i, q, q) - eri(prob, a, q, q, i) for q in range(L) if (sk >> q) & 1)
        return dict(single=True, i=i, a=a, neg=neg, om=other_range(spin, lo, hi), val=v)
    hs = [p for p in range(L) if (hole >> p) & 1]
    ps = [p for p in range(L) if (part >> p) & 1]
    i, j, a, b = hs[0], hs[1], ps[0], ps[1]
    par, m = 0, 0
    for x, y in ((i, a), (j, b)):
        lo, hi = min(x, y), max(x, y)
        par += popc(sk & rmask(lo, hi)) + ((sk >> lo) & 1)
        m ^= other_range(spin, lo, hi)
    if a > j or b < i:
        par += 1
    return dict(single=False, neg=par & 1, om=m, val=eri(prob, a, i, b, j) - eri(prob, a, j, b, i))


def same_spin_element(prob, spin, sr, sk, other):
    e = entry(prob, spin, sr, sk)
    v = e["val"]
    if e["single"]:
        v += sum(eri(prob, e["a"], e["i"], q, q) for q in range(prob.L) if (other >> q) & 1)
    neg = e["neg"] ^ (popc(other & e["om"]) & 1)
    # the parity-table form: xor of prefix parities at the range boundaries
    pp = lambda x: popc(other & rmask(0, x)) & 1  # noqa: E731
    bounds = []
    if e["single"]:
        bounds = [min(e["i"], e["a"]) + spin, max(e["i"], e["a"]) + spin]
    else:
        hole, part = sk & ~sr, sr & ~sk
        hs = [p for p in range(64) if (hole >> p) & 1]
        ps = [p for p in range(64) if (part >> p) & 1]
        for x, y in ((hs[0], ps[0]), (hs[1], ps[1])):
            bounds += [min(x, y) + spin, max(x, y) + spin]
    table_neg = e["neg"]
    for x in bounds:
        table_neg ^= pp(x)
    assert table_neg == neg
    return -v if neg else v


def ab_element(prob, ia_s, ib_s, ja_s, jb_s):
    """Alpha single x beta single as the alpha-beta kernels evaluate it."""
    ea = entry(prob, 0, ia_s, ja_s)
    eb = entry(prob, 1, ib_s, jb_s)
    lo_b, hi_b = min(eb["i"], eb["a"]), max(eb["i"], eb["a"])
    P = prefix_parity(ja_s)
    neg = ea["neg"] ^ (popc(ib_s & ea["om"]) & 1) ^ eb["neg"] ^ (((P >> hi_b) ^ (P >> lo_b)) & 1)
    v = eri(prob, ea["a"], ea["i"], eb["a"], eb["i"])
    return -v if neg else v


@pytest.mark.parametrize("spec", [(8, 3, 2, 40, 25, 3), (12, 4, 4, 60, 60, 5), (16, 2, 5, 30, 80, 9),
                                  (64, 3, 3, 40, 40, 11)])
def test_kernel_algebra_equals_reference_rules(spec):
    L, na_el, nb_el, Na, Nb, seed = spec
    prob = synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)
    port = Port()
    a = [int(x) for x in prob.alpha]
    b = [int(x) for x in prob.beta]
    rng = np.random.default_rng(seed)
    n_checked = 0
    for _ in range(300):
        x, y = int(rng.integers(prob.na)), int(rng.integers(prob.nb))
        for z in range(prob.na):  # alpha excitations, same beta
            d = popc(a[x] ^ a[z])
            if d in (2, 4):
                ref = port.hij(prob, a[x], b[y], a[z], b[y])
                assert abs(same_spin_element(prob, 0, a[x], a[z], b[y]) - ref) <= 1e-12
                n_checked += 1
        for w in range(prob.nb):  # beta excitations, same alpha
            d = popc(b[y] ^ b[w])
            if d in (2, 4):
                ref = port.hij(prob, a[x], b[y], a[x], b[w])
                assert abs(same_spin_element(prob, 1, b[y], b[w], a[x]) - ref) <= 1e-12
                n_checked += 1
        for z in range(prob.na):  # alpha single x beta single
            if popc(a[x] ^ a[z]) != 2:
                continue
            for w in range(prob.nb):
                if popc(b[y] ^ b[w]) != 2:
                    continue
                ref = port.hij(prob, a[x], b[y], a[z], b[w])
                assert abs(ab_element(prob, a[x], b[y], a[z], b[w]) - ref) <= 1e-12
                n_checked += 1
        if n_checked > 6000:
            break
    assert n_checked > 500


def basis_phase(alpha_s, beta_s):
    """phi(alpha, beta) of the alpha-first ordering: the parity of the number of
    (alpha p, beta q) pairs with q < p, up to the basis-wide constant
    (-1)^{n_alpha n_beta}; equal to parity(beta & prefix_parity(alpha))."""
    return popc(beta_s & prefix_parity(alpha_s)) & 1


def separated_element(prob, spin_pairs):
    """H_IJ in the alpha-first ordering, where every sign is a pure same-spin
    sign: ((spin, bra, ket), ...) for the excited spins, plus the opposite-spin
    string of a same-spin excitation for the single's Coulomb term."""
    if len(spin_pairs) == 2:  # alpha single x beta single
        (_, ia_s, ja_s), (_, ib_s, jb_s) = spin_pairs
        ea = entry(prob, 0, ia_s, ja_s)
        eb = entry(prob, 1, ib_s, jb_s)
        v = eri(prob, ea["a"], ea["i"], eb["a"], eb["i"])
        return -v if ea["neg"] ^ eb["neg"] else v
    ((spin, sr, sk, other),) = spin_pairs
    e = entry(prob, spin, sr, sk)
    v = e["val"]
    if e["single"]:  # the opposite-spin Coulomb table entry D[pq(a,i)][other]
        v += sum(eri(prob, e["a"], e["i"], q, q) for q in range(prob.L) if (other >> q) & 1)
    return -v if e["neg"] else v


@pytest.mark.parametrize("spec", [(8, 3, 2, 40, 25, 3), (12, 4, 4, 60, 60, 5), (16, 2, 5, 30, 80, 9),
                                  (64, 3, 3, 40, 40, 11)])
def test_alpha_first_basis_factorises_signs(spec):
    """H_int[I,J] = phi(I) phi(J) H_sep[I,J]: the interleaved matrix elements of
    the reference are the alpha-first ones conjugated by the +-1 basis phase,
    and in the alpha-first basis the opposite-spin string enters no sign."""
    L, na_el, nb_el, Na, Nb, seed = spec
    prob = synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)
    port = Port()
    a = [int(x) for x in prob.alpha]
    b = [int(x) for x in prob.beta]
    rng = np.random.default_rng(seed + 100)
    n_checked = 0

    def check(x, y, z, w, pairs):
        nonlocal n_checked
        ref = port.hij(prob, a[x], b[y], a[z], b[w])
        flip = basis_phase(a[x], b[y]) ^ basis_phase(a[z], b[w])
        sep = separated_element(prob, pairs)
        assert abs((-sep if flip else sep) - ref) <= 1e-12
        n_checked += 1

    for _ in range(300):
        x, y = int(rng.integers(prob.na)), int(rng.integers(prob.nb))
        for z in range(prob.na):
            if popc(a[x] ^ a[z]) in (2, 4):
                check(x, y, z, y, [(0, a[x], a[z], b[y])])
        for w in range(prob.nb):
            if popc(b[y] ^ b[w]) in (2, 4):
                check(x, y, x, w, [(1, b[y], b[w], a[x])])
        for z in range(prob.na):
            if popc(a[x] ^ a[z]) != 2:
                continue
            for w in range(prob.nb):
                if popc(b[y] ^ b[w]) == 2:
                    check(x, y, z, w, [(0, a[x], a[z]), (1, b[y], b[w])])
        if n_checked > 6000:
            break
    assert n_checked > 500


def bit_reverse64(x):
    return int(format(int(x), "064b")[::-1], 2)


@pytest.mark.parametrize("spec", [(12, 4, 4, 81, 60, 5), (16, 3, 5, 50, 70, 9)])
def test_bit_reversed_blocks_reproduce_same_spin_doubles(spec):
    """The blocked same-spin kernel's decomposition: bra strings ordered by
    their bit-reversed words and cut into blocks of 4; per block the union of
    the 4 strings' double-excitation kets (ascending) with a dense 4 x |union|
    matrix of signed same-spin values (zero where a string does not connect).
    Block-by-block products must reproduce the per-string products of the
    reference lists (the oracle's connectivity, doubles ascending per row)."""
    L, na_el, nb_el, Na, Nb, seed = spec
    prob = synth.random_problem(L, na_el, nb_el, Na, Nb, seed=seed)
    port = Port()
    a = [int(x) for x in prob.alpha]
    sl, dl, idx = port.connectivity(prob.alpha)
    off = np.concatenate([[0], np.cumsum(sl.astype(np.int64) + dl.astype(np.int64))])
    dbl = [idx[off[r] + int(sl[r]):off[r + 1]].astype(np.int64) for r in range(Na)]
    for d in dbl:  # the builder merges rows whose doubles are ascending
        assert np.all(np.diff(d) > 0)
    val = {}
    for r in range(Na):
        for k in dbl[r]:
            e = entry(prob, 0, a[r], a[int(k)])
            val[(r, int(k))] = -e["val"] if e["neg"] else e["val"]
    X = np.random.default_rng(seed).standard_normal((Na, Nb))
    ref = np.zeros((Na, Nb))
    for r in range(Na):
        for k in dbl[r]:
            ref[r] += val[(r, int(k))] * X[int(k)]
    order = sorted(range(Na), key=lambda r: bit_reverse64(a[r]))
    out = np.full((Na, Nb), np.nan)
    for b0 in range(0, Na, 4):
        rows = order[b0:b0 + 4]
        union = sorted(set(int(k) for r in rows for k in dbl[r]))
        V = np.zeros((len(rows), len(union)))
        pos = {k: t for t, k in enumerate(union)}
        for i, r in enumerate(rows):
            for k in dbl[r]:
                V[i, pos[int(k)]] = val[(r, int(k))]
        out[rows] = V @ X[union] if union else 0.0
    assert np.abs(out - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_bit_reversed_order_shares_more_kets_than_ascending():
    """Why the blocks use bit-reversed order: on the 400-string sample of the
    24-orbital workload, four bit-reversed neighbours share more of their
    double-excitation kets than four neighbours in ascending order."""
    prob = synth.config("cfg1")
    port = Port()
    sl, dl, idx = port.connectivity(prob.alpha)
    off = np.concatenate([[0], np.cumsum(sl.astype(np.int64) + dl.astype(np.int64))])
    dbl = [idx[off[r] + int(sl[r]):off[r + 1]] for r in range(prob.na)]

    def ratio(order):
        tot = uni = 0
        for b0 in range(0, len(order), 4):
            seg = np.concatenate([dbl[r] for r in order[b0:b0 + 4]])
            tot += len(seg)
            uni += len(np.unique(seg))
        return uni / tot

    rev = sorted(range(prob.na), key=lambda r: bit_reverse64(prob.alpha[r]))
    assert ratio(rev) < ratio(list(range(prob.na)))
