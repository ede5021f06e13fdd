"""Host logic of the multi-GPU runs, on CPU: the ensemble partition and the rank
reductions, with two gloo ranks (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def test_partition_covers_all_members_and_balances_cost():
    from mcstar_b200 import ensemble_members, partition, member_cost
    members = ensemble_members(seed=4)
    assert len(members) == 64
    assert sum(1 for m in members if m["shape"][2] == 1) == 48
    for n in (1, 2, 4, 8):
        parts = partition(members, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(member_cost(members[i]) for i in p) for p in parts]
        biggest = max(member_cost(m) for m in members)
        assert max(loads) - min(loads) <= biggest + 1e-6
    assert partition(members, 4) == partition(members, 4)


def test_ensemble_members_ranges():
    from mcstar_b200 import ensemble_members
    from mcstar_b200.ensemble import SIDES_2D, SIDES_3D
    for m in ensemble_members(seed=9):
        nx, ny, nz = m["shape"]
        assert nx == ny and (nz == 1 and nx in SIDES_2D or nz == nx and nx in SIDES_3D)
        assert 0.1 <= m["eps"] <= 0.4 and -0.35 <= m["psi0"] <= -0.15


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mcstar-libs_b200"))
    from mcstar_b200 import dist, ensemble_members, partition
    w, r, _ = dist.env_world()
    dist.init("gloo", timeout_s=60)
    members = ensemble_members(seed=4)
    mine = partition(members, w)[r]
    cells = sum(members[i]["shape"][0] * members[i]["shape"][1] * members[i]["shape"][2] for i in mine)
    fake_ms = 10.0 + r  # a rank's device time
    dist.barrier(w)
    ms_max, = dist.reduce_scalars(w, [fake_ms], "max")
    total_cells, nmem = dist.reduce_scalars(w, [cells, len(mine)], "sum")
    q.put((r, ms_max, total_cells, nmem))
    dist.shutdown(w)


def test_two_gloo_ranks_shard_members_and_reduce_scalars():
    from mcstar_b200 import ensemble_members
    members = ensemble_members(seed=4)
    all_cells = sum(m["shape"][0] * m["shape"][1] * m["shape"][2] for m in members)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ms_max, total_cells, nmem in res:
        assert ms_max == 11.0
        assert total_cells == all_cells
        assert nmem == 64
