"""Session sharding across GPUs (one process per GPU, no data-path exchange).

Sessions are independent -- each owns its IR spectra, delay line and history
-- so the multi-GPU form is a router: every session is placed on one rank and
stays there. Placement balances the per-block HBM traffic of the tail
(16 bytes x channels x (partitions - 1) x block, the MAC's algorithmic bytes)
subject to each rank's device-memory budget. The control plane (who serves
which session) is decided on rank 0 and broadcast; audio never crosses GPUs.
"""
from __future__ import annotations

import dataclasses
import heapq


@dataclasses.dataclass(frozen=True)
class SessionSpec:
    sid: int
    channels: int
    ir_length: int


def partitions(ir_length: int, block: int) -> int:
    return max(1, -(-ir_length // block))


def tail_bytes(s: SessionSpec, block: int) -> int:
    """Algorithmic HBM bytes per block of the session's tail MAC (FP32 spectra)."""
    return 16 * s.channels * (partitions(s.ir_length, block) - 1) * block


def device_bytes(s: SessionSpec, block: int) -> int:
    """Resident bytes of the session on its GPU (two IR slots, delay line, history)."""
    P = partitions(s.ir_length, block)
    return s.channels * (2 * P * block * 8 + P * block * 8 + block * 4)


def assign(sessions, n_ranks: int, block: int, budget_bytes: int | None = None):
    """Greedy longest-first placement on the least-loaded rank that has room.

    Returns {sid: rank}; sessions that fit nowhere map to -1 (refused)."""
    order = sorted(sessions, key=lambda s: (-tail_bytes(s, block), s.sid))
    heap = [(0, r) for r in range(n_ranks)]
    mem = [0] * n_ranks
    out = {}
    for s in order:
        need = device_bytes(s, block)
        popped = []
        placed = -1
        while heap:
            load, r = heapq.heappop(heap)
            if budget_bytes is None or mem[r] + need <= budget_bytes:
                mem[r] += need
                heapq.heappush(heap, (load + tail_bytes(s, block), r))
                placed = r
                break
            popped.append((load, r))
        for item in popped:
            heapq.heappush(heap, item)
        out[s.sid] = placed
    return out


def loads(sessions, placement, n_ranks: int, block: int):
    per = [0] * n_ranks
    for s in sessions:
        r = placement[s.sid]
        if r >= 0:
            per[r] += tail_bytes(s, block)
    return per


def broadcast_placement(pg, sessions, block: int, budget_bytes: int | None = None):
    """Rank 0 decides, every rank receives the same placement (torch.distributed)."""
    world = pg.get_world_size()
    obj = [assign(sessions, world, block, budget_bytes) if pg.get_rank() == 0 else None]
    pg.broadcast_object_list(obj, src=0)
    return obj[0]
