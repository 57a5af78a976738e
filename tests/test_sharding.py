"""Multi-GPU control plane on CPU: session placement and the per-rank loop,
run as world_size-2 gloo process groups (no GPU). Also checks that a rank
failing mid-run ends the others with an error instead of a hang."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from tan_b200 import sharding as sh


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sessions(n=60, seed=5):
    g = np.random.Generator(np.random.PCG64(seed))
    return [sh.SessionSpec(i, int(g.integers(1, 9)), int(np.exp(g.uniform(np.log(8192), np.log(524288)))))
            for i in range(n)]


def test_placement_is_complete_and_balanced():
    ss = _sessions()
    pl = sh.assign(ss, 4, 256)
    assert sorted(pl) == [s.sid for s in ss]
    assert all(0 <= r < 4 for r in pl.values())
    per = sh.loads(ss, pl, 4, 256)
    assert max(per) / min(per) < 1.15


def test_placement_respects_memory_budget():
    ss = _sessions(40)
    total = sum(sh.device_bytes(s, 256) for s in ss)
    budget = total // 3  # two ranks cannot hold everything
    pl = sh.assign(ss, 2, 256, budget)
    used = [0, 0]
    for s in ss:
        if pl[s.sid] >= 0:
            used[pl[s.sid]] += sh.device_bytes(s, 256)
    assert max(used) <= budget
    assert any(r == -1 for r in pl.values())


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        ss = _sessions(30, seed=9)
        pl = sh.broadcast_placement(dist, ss, 256)
        mine = [s for s in ss if pl[s.sid] == rank]
        # per-rank work of one block (stand-in for the engine): bytes of its shard
        t = torch.tensor([float(sum(sh.tail_bytes(s, 256) for s in mine))], dtype=torch.float64)
        if mode == "fail" and rank == 1:
            raise RuntimeError("injected failure on rank 1 before the reduction")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        q.put((rank, sorted(s.sid for s in mine), float(t.item()), None))
    except Exception as e:  # noqa: BLE001
        q.put((rank, None, None, type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(out)


def test_two_rank_placement_covers_every_session_once():
    out = _run("ok")
    (r0, s0, m0, e0), (r1, s1, m1, e1) = out
    assert e0 is None and e1 is None
    assert sorted(s0 + s1) == list(range(30)) and not set(s0) & set(s1)
    assert m0 == m1 > 0


def test_failed_rank_ends_peers_with_an_error():
    out = _run("fail")
    errs = {r: e for r, _, _, e in out}
    assert errs[1] == "RuntimeError"
    assert errs[0] is not None  # the peer's collective failed or timed out, it did not hang


class FakeEngine:
    """Stand-in for a rank's engine on CPU: a byte budget (the engine's own
    session size rule) and a set of sessions it refuses (as a fragmented arena
    or a full slot table would)."""

    def __init__(self, budget, refuse=()):
        self.budget, self.used, self.refuse, self.open_ids = budget, 0, set(refuse), set()
        self.blocks = {}

    def open(self, spec):
        need = sh.device_bytes(spec, 256)
        if spec.sid in self.refuse or self.used + need > self.budget:
            return None
        self.used += need
        self.open_ids.add(spec.sid)
        return (spec.sid, need)

    def close(self, handle):
        self.used -= handle[1]
        self.open_ids.discard(handle[0])

    # session state: blocks served, carried by a handover
    def tick(self, handles):
        for h in handles:
            self.blocks[h[0]] = self.blocks.get(h[0], 0) + 1

    def snapshot(self, handle):
        return f"{handle[0]}:{self.blocks.get(handle[0], 0)}".encode()

    def restore(self, spec, blob):
        sid, blocks = (int(v) for v in bytes(blob).decode().split(":"))
        assert sid == spec.sid
        h = self.open(spec)
        if h is not None:
            self.blocks[sid] = blocks
        return h


def _server_worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import time

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        store = dist.distributed_c10d._get_default_store()
        ss = _sessions(24, seed=11)
        budget = sum(sh.device_bytes(s, 256) for s in ss)  # either rank could hold everything
        refuse = {s.sid for s in ss[:5]} if rank == 1 else set()
        srv = sh.RankServer(dist, FakeEngine(budget, refuse), 256, budget, store)
        pl = srv.place(ss)
        mine_first = sorted(srv.handles)
        taken = []
        if mode in ("leave", "handover"):
            for k in range(200):  # blocks
                if rank == 1 and k == 3:
                    srv.leave(handover=(mode == "handover"))
                    break
                if rank == 0:
                    taken += srv.check_peers()
                    if srv.left:
                        break
                srv.engine.tick(srv.handles.values())
                time.sleep(0.01)
        states = {sid: srv.engine.blocks.get(sid, 0) for sid in taken}
        q.put((rank, pl, mine_first, sorted(srv.engine.open_ids), taken, None, sorted(srv.restored), states))
    except Exception as e:  # noqa: BLE001
        q.put((rank, None, None, None, None, repr(e), None, None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run_server(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_server_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_rank_server_replaces_refused_sessions_on_the_other_rank():
    (r0, pl0, m0, open0, _, e0, _, _), (r1, pl1, m1, open1, _, e1, _, _) = _run_server("ok")
    assert e0 is None and e1 is None, (e0, e1)
    assert pl0 == pl1  # every rank holds the same placement
    ss = _sessions(24, seed=11)
    assert sorted(pl0) == [s.sid for s in ss] and all(r in (0, 1) for r in pl0.values())
    assert all(pl0[s.sid] == 0 for s in ss[:5])  # refused by rank 1, re-placed on rank 0
    assert sorted(m0 + m1) == sorted(s.sid for s in ss) and not set(m0) & set(m1)
    assert set(m0) == {sid for sid, r in pl0.items() if r == 0}


def test_rank_leaving_between_blocks_hands_its_sessions_over():
    (r0, pl0, m0, open0, taken, e0, restored, _), (r1, pl1, m1, open1, _, e1, _, _) = _run_server("leave")
    assert e0 is None and e1 is None, (e0, e1)
    assert m1 and open1 == []  # rank 1 closed its sessions when it left
    assert sorted(taken) == sorted(m1)  # rank 0 took every one of them over
    assert sorted(open0) == sorted(m0 + m1)
    assert restored == []  # opened afresh: no state was handed over


def test_rank_leaving_with_handover_passes_each_sessions_state():
    (r0, pl0, m0, open0, taken, e0, restored, states), (r1, _, m1, open1, _, e1, _, _) = _run_server("handover")
    assert e0 is None and e1 is None, (e0, e1)
    assert sorted(taken) == sorted(m1) and open1 == []
    assert restored == sorted(m1)  # every one restored from its state
    assert all(states[sid] == 3 for sid in m1), states  # the blocks rank 1 had served them


def test_device_bytes_follow_the_engine_rule_for_non_uniform_sessions():
    u = sh.SessionSpec(0, 2, 1 << 20)
    n = sh.SessionSpec(1, 2, 1 << 20, ((256, 2), (512, 2), (1024, 2), (2048, 2), (4096, 2), (8192, 2), (16384, 63)))
    assert sh.device_bytes(n, 256) > 0 and sh.device_bytes(u, 256) > 0
    assert sh.tail_bytes(n, 256) < sh.tail_bytes(u, 256) / 8  # the levels stream far fewer bytes per block
