"""Alpha-row shards of the solve over several ranks (sbdx/shard.py), on the
CPU with gloo at world size 2.

The host logic of the multi-GPU path is exercised with the oracle standing
in for each rank's row-range product (on a GPU that is
sbdx_sigma_rows_device): the row partition, the variable-size gather of the
whole vector, the all-reduced dots and the redundant Rayleigh-Ritz step. The
sharded FP64 Davidson must give the single-process oracle's energy within
1e-9 Ha and the same vector, on every rank."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPEC = (14, 4, 4, 90, 70, 21)  # L, alpha and beta electrons, Na, Nb, seed


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def oracle_work(port, prob):
    sa, da, _ = port.connectivity(prob.alpha)
    sb, db, _ = port.connectivity(prob.beta)
    return (sa + da).astype(float) * prob.nb + sa.astype(float) * float(sb.sum()) + float((sb + db).sum())


def worker(rank, world, port_no, out):
    import sys

    for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "sbd-ykt_b200")):
        sys.path.insert(0, p)
    from oracle import Port
    from sbdx import shard, synth

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port_no))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = synth.random_problem(*SPEC)
        port = Port()
        nb, D = prob.nb, prob.D
        hii = torch.from_numpy(port.diag_terms(prob))
        bounds = shard.partition(oracle_work(port, prob), world)
        comm = shard.Comm(dist.group.WORLD)
        a0, a1 = bounds[rank]
        full = torch.zeros(D, dtype=torch.float64)
        hii_loc = hii[a0 * nb:a1 * nb].clone()

        def apply(x, y):
            comm.gather_rows(full, x, bounds, nb)
            off = port.sigma_rows(prob, full.numpy(), a0, a1 - a0) if a1 > a0 else np.zeros(0)
            y.copy_(torch.from_numpy(off) + hii_loc * x)

        W0 = torch.zeros(D, dtype=torch.float64)
        W0[0] = 1.0
        E, W, info = shard.davidson(apply, hii_loc, comm, W0[a0 * nb:a1 * nb].clone(), max_it=6, max_nb=10, eps=1e-9)
        Wfull = torch.zeros(D, dtype=torch.float64)
        comm.gather_rows(Wfull, W, bounds, nb)
        out[rank] = (E, info["sigmas"], info["residual"], bounds, Wfull.numpy().copy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_davidson_matches_single_process_over_gloo():
    import sys

    sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "sbd-ykt_b200")]
    from oracle import Port
    from sbdx import synth

    world = 2
    port_no = free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(worker, args=(world, port_no, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    prob = synth.random_problem(*SPEC)
    E_ref, W_ref, _ = Port().davidson(prob, max_it=6, max_nb=10, eps=1e-9)
    assert set(res) == {0, 1}
    (E0, n0, r0, b0, W0), (E1, n1, r1, b1, W1) = res[0], res[1]
    assert b0 == b1 and b0[0][0] == 0 and b0[-1][1] == prob.na and b0[0][1] == b0[1][0]
    assert 0 < b0[0][1] < prob.na  # both ranks own rows
    assert E0 == E1 and n0 == n1 and r0 == r1  # every rank takes the same steps
    assert abs(E0 - E_ref) < 1e-9
    assert abs(abs(np.dot(W0, W_ref)) - 1.0) < 1e-8
    assert np.array_equal(W0, W1)


def test_partition_blocks():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "sbd-ykt_b200"))
    from sbdx import shard

    rng = np.random.default_rng(3)
    for n in (7, 64, 1000, 8003):
        work = rng.random(n) * 10
        for world in (1, 2, 3, 8):
            b = shard.partition(work, world)
            assert len(b) == world and b[0][0] == 0 and b[-1][1] == n
            for (x0, x1), (y0, _) in zip(b, b[1:]):
                assert x1 == y0 and x0 <= x1
            for x0, x1 in b:
                assert x0 % 8 == 0 or x0 == x1
            if n >= 64 * world:  # balanced to within a few rows' work
                sums = [work[x0:x1].sum() for x0, x1 in b]
                assert max(sums) - min(sums) < 16 * work.max()
