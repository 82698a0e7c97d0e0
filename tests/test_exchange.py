"""Multi-process halo exchange on CPU ranks (gloo, world size 2 and 3):
every process holds the whole arena with only its own blocks' points known;
after ExchangePlan.exchange, every source of its own blocks' halo program
(cc_halo_dependencies) holds the owner's value, and nothing else was
written.  The dependency query and the arena layout need no device."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from combustioncodegpu_b200 import cases

    # 2 x 2 x 1 blocks of uneven sizes, periodic, 9 species
    return cases.case_multiblock(([6, 7], [6, 5], [5]), species=cases.synthetic_species())


def _spans(d, nb):
    return np.array([d.block_arena(b) for b in range(nb)], dtype=np.int64)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import exchange

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    case = _case()
    d = cc.Driver.from_case(case, "mixed")
    nb = len(case["blocks"])
    spans = _spans(d, nb)
    owner = exchange.partition([int(c) for c in spans[:, 1]], world)
    plan = exchange.ExchangePlan(d, owner, rank, world)
    n = int((spans[:, 0] + spans[:, 1]).max())
    rng = np.random.default_rng(5)
    truth = [[rng.standard_normal(n) for _ in range(3)] for _ in range(2)]  # [state][field]
    mine = np.zeros(n, dtype=bool)
    for b in range(nb):
        if owner[b] == rank:
            mine[spans[b, 0]:spans[b, 0] + spans[b, 1]] = True
    states = [[torch.from_numpy(np.where(mine, t, np.nan)) for t in fields] for fields in truth]
    before = [[f.clone() for f in fields] for fields in states]
    plan.exchange(states)
    dst, src, which = d.halo_dependencies()
    own_dst = mine[dst]
    ok_sources = all(
        np.array_equal(states[w][f].numpy()[src[own_dst & (which == w)]], truth[w][f][src[own_dst & (which == w)]])
        for w in (0, 1) for f in range(3))
    # written points: exactly the received ones
    received = [np.zeros(n, dtype=bool) for _ in range(2)]
    for q in plan.recv:
        for w in (0, 1):
            received[w][plan.recv[q][w]] = True
    untouched = all(
        np.array_equal(np.isnan(states[w][f].numpy()), np.isnan(before[w][f].numpy()) & ~received[w])
        for w in (0, 1) for f in range(3))
    sent, got = plan.volume()
    d.close()
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out, "rank%d.npy" % rank), np.array([ok_sources, untouched, sent, got], dtype=np.int64))


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_delivers_every_halo_source(tmp_path, world):
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [np.load(tmp_path / ("rank%d.npy" % r)) for r in range(world)]
    for r, (ok, untouched, sent, got) in enumerate(res):
        assert ok == 1, "rank %d: a halo source differs from its owner's value" % r
        assert untouched == 1, "rank %d: points other than the received ones were written" % r
        assert got > 0, "rank %d received nothing: the partition has no cross-process interface" % r
    assert sum(int(x[2]) for x in res) == sum(int(x[3]) for x in res)  # every point sent is received


def test_partition_and_single_process_plan():
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import exchange

    # largest first to the lighter rank: 40 -> 0, 30 -> 1, 20 -> 1, 10 -> 0 (loads 50 / 50)
    assert exchange.partition([10, 40, 20, 30], 2) == [0, 0, 1, 1]
    owner = exchange.partition([5, 5, 5, 5, 5], 3)
    assert sorted(np.bincount(owner, minlength=3)) == [1, 2, 2]
    case = _case()
    d = cc.Driver.from_case(case, "mixed")
    plan = exchange.ExchangePlan(d, [0] * len(case["blocks"]), 0, 1)
    assert plan.volume() == (0, 0) and plan.send == {} and plan.recv == {}
    d.close()


def _step_worker(rank, world, port, out, precision):
    import torch.distributed as dist

    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import exchange

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    case = _case()
    d = cc.Driver.from_case(case, precision)
    nb = len(case["blocks"])
    owner = exchange.partition([int(c) for c in _spans(d, nb)[:, 1]], world)
    step = exchange.DistributedStep(d, owner, rank, world)
    d.initialize_computation()
    d.simulate(3, "rk3", residual=True)
    res = step.residual()
    dt = d.last_dt()
    status = d.status()
    states = {b: d.field[b].get_state()[2] for b in range(nb) if owner[b] == rank}
    step.close()
    d.close()
    dist.barrier()
    dist.destroy_process_group()
    np.savez(os.path.join(out, "step%d.npz" % rank), res=res, dt=dt, status=status, owner=np.array(owner),
             **{"b%d" % b: v for b, v in states.items()})


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_process_step_equals_single_process(tmp_path, precision):
    """Two processes on one GPU (gloo between them, the exchange on the host
    between launches, so no kernel waits on another process), each advancing
    its own blocks of the 2 x 2 x 1 periodic multiblock case for three RK3
    steps with the halo sources exchanged inside cc_step and the time step
    reduced over processes: every block's state equals the single-process
    run's bit for bit, the residual to rounding (its sums are added in
    another order)."""
    import combustioncodegpu_b200 as cc

    world = 2
    mp.spawn(_step_worker, args=(world, _free_port(), str(tmp_path), precision), nprocs=world, join=True)
    case = _case()
    d = cc.Driver.from_case(case, precision)
    d.initialize_computation()
    d.simulate(3, "rk3", residual=True)
    want = [d.field[b].get_state()[2] for b in range(len(case["blocks"]))]
    want_res, want_dt = d.residual(), d.last_dt()
    assert d.status() == 0
    d.close()
    got = [np.load(tmp_path / ("step%d.npz" % r)) for r in range(world)]
    owner = got[0]["owner"]
    assert set(owner.tolist()) == {0, 1}
    for b in range(len(case["blocks"])):
        np.testing.assert_array_equal(got[owner[b]]["b%d" % b], want[b])
    for g in got:
        assert int(g["status"]) == 0
        assert float(g["dt"]) == want_dt
        np.testing.assert_allclose(g["res"], want_res, rtol=1e-12)
