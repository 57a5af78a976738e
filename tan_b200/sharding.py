"""Session sharding across GPUs (one process per GPU, no data-path exchange).

Sessions are independent -- each owns its IR spectra, delay line and history
-- so the multi-GPU form is a router: every session is placed on one rank and
stays there. Placement balances the per-block HBM traffic of the tail (the
MAC's algorithmic bytes) subject to each rank's device-memory budget, counted
with the engine's own admission rule (tanb_engine_session_bytes, so a rank's
engine never refuses a placement that fits its budget for lack of bytes). The
control plane (who serves which session) is decided on rank 0 and broadcast;
audio never crosses GPUs.

RankServer runs the control plane on every rank: the initial placement, the
re-placement of sessions a rank's engine refused (on the ranks that did not
refuse them), and, between blocks, the take-over of the sessions of a rank that
left (announced through the process group's store, so the others learn it on
the host before their next block and no collective is pending when it goes),
optionally with each session's state handed over so that its audio continues.
"""
from __future__ import annotations

import dataclasses
import heapq


@dataclasses.dataclass(frozen=True)
class SessionSpec:
    sid: int
    channels: int
    ir_length: int
    levels: tuple | None = None  # non-uniform schedule ((block, partitions), ...) or None


def partitions(ir_length: int, block: int) -> int:
    return max(1, -(-ir_length // block))


def tail_bytes(s: SessionSpec, block: int) -> int:
    """Algorithmic HBM bytes per block of the session's tail MAC (FP32
    spectra): uniform sessions stream partitions [1, P) of IR spectrum and
    delay line every block; a non-uniform level of block N and K partitions
    streams its partitions [1, K) once per N / block blocks."""
    if not s.levels:
        return 16 * s.channels * (partitions(s.ir_length, block) - 1) * block
    total = 0
    for N, K in s.levels:
        total += 16 * (K - 1) * N * block // N
    return s.channels * total


def device_bytes(s: SessionSpec, block: int, spectrum: int = 0) -> int:
    """Device bytes the session takes from an engine's budget (the engine's own
    arena rule: IR spectra in two slots, delay lines, history, partial sums,
    and for non-uniform sessions their level rings and input history)."""
    from . import engine as eng

    return eng.session_bytes(block, s.channels, s.ir_length, list(s.levels) if s.levels else None, spectrum)


def assign(sessions, n_ranks: int, block: int, budget_bytes: int | None = None, used=None, exclude=None,
           ranks=None):
    """Greedy longest-first placement on the least-loaded rank that has room.

    used: bytes already in use per rank (default 0); exclude: {sid: set of
    ranks that must not take it}; ranks: the ranks that may take sessions
    (default all). Returns {sid: rank}; sessions that fit nowhere map to -1."""
    ranks = list(range(n_ranks)) if ranks is None else list(ranks)
    exclude = exclude or {}
    order = sorted(sessions, key=lambda s: (-tail_bytes(s, block), s.sid))
    mem = list(used) if used is not None else [0] * n_ranks
    heap = [(0, r) for r in ranks]
    out = {}
    for s in order:
        need = device_bytes(s, block)
        popped = []
        placed = -1
        while heap:
            load, r = heapq.heappop(heap)
            if r not in exclude.get(s.sid, ()) and (budget_bytes is None or mem[r] + need <= budget_bytes):
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


class RankServer:
    """The per-rank control plane of sharded serving.

    engine: this rank's engine, an object with open(spec) -> handle or None
    (refused) and close(handle). pg: torch.distributed (gloo or nccl); store:
    the process group's key-value store, for the leave announcements."""

    def __init__(self, pg, engine, block: int, budget_bytes: int | None, store=None):
        self.pg, self.engine, self.block, self.budget = pg, engine, block, budget_bytes
        self.rank, self.world = pg.get_rank(), pg.get_world_size()
        self.store = store
        self.placement = {}
        self.handles = {}  # sid -> engine handle of the sessions this rank serves
        self.sessions = {}
        self.left = set()
        self.restored = []  # sids taken over with their state (leave(handover=True))

    def place(self, sessions, rounds: int | None = None):
        """Places `sessions` over the live ranks; sessions a rank's engine
        refuses are re-placed on ranks that did not refuse them. Returns the
        final placement ({sid: rank}, -1 when no rank could take one)."""
        for s in sessions:
            self.sessions[s.sid] = s
        live = [r for r in range(self.world) if r not in self.left]
        pending = list(sessions)
        exclude = {}
        for _ in range(rounds or self.world):
            if not pending:
                break
            used = [0] * self.world
            for sid, r in self.placement.items():
                if r >= 0:
                    used[r] += device_bytes(self.sessions[sid], self.block)
            obj = [assign(pending, self.world, self.block, self.budget, used, exclude, live)
                   if self.rank == 0 else None]
            self.pg.broadcast_object_list(obj, src=0)
            new = obj[0]
            refused = []
            for s in pending:
                if new[s.sid] != self.rank:
                    continue
                h = self.engine.open(s)
                if h is None:
                    refused.append(s.sid)
                else:
                    self.handles[s.sid] = h
            lists = [None] * self.world
            self.pg.all_gather_object(lists, refused)
            refused_all = {sid: r for r, lst in enumerate(lists) for sid in (lst or [])}
            for sid, r in new.items():
                if sid not in refused_all:
                    self.placement[sid] = r
            for sid, r in refused_all.items():
                exclude.setdefault(sid, set()).add(r)
            pending = [self.sessions[sid] for sid in refused_all]
        for s in pending:
            self.placement[s.sid] = -1
        return dict(self.placement)

    def leave(self, handover: bool = False):
        """This rank stops between blocks: it closes its sessions and announces
        it; the other ranks take its sessions over before their next block.
        With handover, each session's state (engine.snapshot) goes into the
        store first, and the rank that takes the session over restores it, so
        that its audio continues instead of restarting from silence. (The store
        carries it here; between GPUs of one node a device-to-device copy
        would.)"""
        if handover and self.store is not None:
            for sid, h in self.handles.items():
                blob = self.engine.snapshot(h) if hasattr(self.engine, "snapshot") else None
                if blob is not None:
                    self.store.set(f"tanb/state/{sid}", blob)
        for h in self.handles.values():
            self.engine.close(h)
        self.handles.clear()
        if self.store is not None:
            self.store.set(f"tanb/left/{self.rank}", "1")

    def check_peers(self):
        """Called between blocks: learns of ranks that left (from the store)
        and opens the sessions of theirs that this rank now serves. The new
        placement is computed the same way on every live rank from the same
        data, so no collective is needed. Returns the sids taken over here."""
        if self.store is None:
            return []
        gone = [r for r in range(self.world) if r != self.rank and r not in self.left
                and self.store.check([f"tanb/left/{r}"])]
        taken = []
        for r in sorted(gone):
            self.left.add(r)
            orphans = [self.sessions[sid] for sid, pr in sorted(self.placement.items()) if pr == r]
            live = [q for q in range(self.world) if q not in self.left]
            used = [0] * self.world
            for sid, pr in self.placement.items():
                if pr >= 0 and pr != r:
                    used[pr] += device_bytes(self.sessions[sid], self.block)
            new = assign(orphans, self.world, self.block, self.budget, used, None, live)
            for s in orphans:
                self.placement[s.sid] = new[s.sid]
                if new[s.sid] == self.rank:
                    key = f"tanb/state/{s.sid}"
                    h = None
                    if hasattr(self.engine, "restore") and self.store.check([key]):
                        h = self.engine.restore(s, self.store.get(key))
                        if h is not None:
                            self.restored.append(s.sid)
                    if h is None:
                        h = self.engine.open(s)
                    if h is not None:
                        self.handles[s.sid] = h
                        taken.append(s.sid)
                    else:
                        self.placement[s.sid] = -1
        return taken
