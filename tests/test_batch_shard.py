"""Multi-GPU ensemble host logic on CPU: the instance partition and the
end-of-run gather, run as two gloo ranks (the ensemble has no collective
inside a step, so these are the only cross-rank operations)."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from core_collapse_b200.batch import gather_by_instance, partition_by_cells
from core_collapse_b200.mhd2d import Params


def _ensemble(n=37, seed=2):
    rng = np.random.default_rng(seed)
    return [Params(Nx=int(s), Ny=int(s)) for s in rng.choice([64, 96, 128, 192, 256], size=n)]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_every_instance_once_and_balances_cells(world):
    params = _ensemble()
    parts = partition_by_cells(params, world)
    flat = sorted(i for pl in parts for i in pl)
    assert flat == list(range(len(params)))
    loads = [sum(params[i].Nx * params[i].Ny for i in pl) for pl in parts]
    biggest = max(p.Nx * p.Ny for p in params)
    assert max(loads) - min(loads) <= biggest
    assert all(pl == sorted(pl) for pl in parts)
    assert partition_by_cells(params, world) == parts   # deterministic


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle_lib as O
        from cases_mhd2d import CASES, make_case
        names = sorted(CASES)
        cases = [make_case(nm) for nm in names]
        params = [c[0] for c in cases]
        mine = partition_by_cells(params, world)[rank]
        local = {}
        for i in mine:
            p, U, B = cases[i]
            local[i] = O.oracle().or_mhd2d_compute_dt(C.byref(p.to_c()), O.pp(O.state_list(U, B)))
        merged = gather_by_instance(local, world)
        q.put((rank, mine, merged))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_instance():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    import oracle_lib as O
    from cases_mhd2d import CASES, make_case
    want = {}
    for i, nm in enumerate(sorted(CASES)):
        p, U, B = make_case(nm)
        want[i] = O.oracle().or_mhd2d_compute_dt(C.byref(p.to_c()), O.pp(O.state_list(U, B)))
    mines = sorted(i for _, mine, _ in got for i in mine)
    assert mines == list(range(len(CASES)))
    for _, _, merged in got:
        assert merged == want
