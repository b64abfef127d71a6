"""Replicas: the search on several GPUs, one process per GPU.

The walkers of a search are independent, so the search shards without a
data-path collective: every rank walks its own seeded walkers on its own GPU,
and after each launch the ranks exchange one small record (found / error, and
the best hit) over the process group, so that all stop together and agree on
one winner.  This is fleet.sh's first-hit-wins mode (fleet.sh:61-123: one
search per machine, stop the rest on the first hit) inside one node, with
torch.distributed as the plumbing.

Determinism: every rank launches the same number of keys per lane each round,
so a round's hits on all ranks cover the same walk indices; the winner is the
hit with the smallest (n, lane, rank), the same whatever the timing.

    python -m torch.distributed.run --nproc-per-node N lxmf-vanity_b200/lxmfv_replicas.py \\
        --seed 7 --aspect lxmf.delivery b00b1

Rank r walks the seeded walkers of seed + RANK_SEED_STRIDE * r (lane 0 its
identity's scalar; lane t the t-th further draw) with that identity's
Ed25519 seed.  Without --seed, each rank draws from the OS.
"""
from __future__ import annotations

import argparse
import datetime
import os
import sys
from dataclasses import dataclass

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lxmfv as lx  # noqa: E402

RANK_SEED_STRIDE = 1000
ST_NONE, ST_FOUND, ST_ERROR = 0, 1, 2


def rank_seed(base: int, rank: int) -> int:
    """The seed of rank `rank`'s walkers: disjoint streams per rank."""
    return base + RANK_SEED_STRIDE * rank


def max_over_ranks(dist, x: float, device: str = "cpu") -> float:
    """The largest `x` over all ranks (device-timed figures are reported as the slowest rank's)."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: float, seconds_max: float, world: int) -> float:
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / seconds_max


@dataclass
class Winner:
    rank: int
    lane: int
    n: int
    identity: bytes


def exchange(dist, status: int, lane: int, n: int, device: str = "cpu") -> list[tuple[int, int, int]]:
    """All ranks' (status, n, lane) records of one round, indexed by rank."""
    import torch
    rec = torch.tensor([status, n, lane], dtype=torch.int64, device=device)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [(status, n, lane)]
    out = [torch.zeros(3, dtype=torch.int64, device=device) for _ in range(dist.get_world_size())]
    dist.all_gather(out, rec)
    return [tuple(int(v) for v in o.tolist()) for o in out]


def pick_winner(records: list[tuple[int, int, int]]) -> int | None:
    """The rank whose hit has the smallest (n, lane, rank), or None."""
    found = [(n, lane, r) for r, (st, n, lane) in enumerate(records) if st == ST_FOUND]
    return min(found)[2] if found else None


def share_identity(dist, identity: bytes | None, src: int, device: str = "cpu") -> bytes:
    """Rank `src`'s 64-byte identity, on every rank."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        assert identity is not None
        return identity
    t = torch.zeros(64, dtype=torch.uint8, device=device)
    if identity is not None:
        t.copy_(torch.frombuffer(bytearray(identity), dtype=torch.uint8))
    dist.broadcast(t, src=src)
    return bytes(t.cpu().numpy().tobytes())


def replicated_search(dist, engine, max_rounds: int, device: str = "cpu") -> Winner | None:
    """Runs `engine` (an object with launch() -> [(lane, n)], identity(lane, n),
    recheck(identity)) round by round on every rank until some rank's hit
    passes its recheck, then returns the common winner on every rank.

    Every rank takes the same collective steps each round, also when its
    engine fails: a failure is reported in the round's record and every rank
    raises, so no rank is left waiting in a collective."""
    rank = dist.get_rank() if dist is not None and dist.is_initialized() else 0
    for _ in range(max_rounds):
        status, lane, n, ident, err = ST_NONE, 0, 0, None, None
        try:
            hits = engine.launch()
            if hits:
                lane, n = min(hits, key=lambda h: (h[1], h[0]))
                ident = engine.identity(lane, n)
                if not engine.recheck(ident):
                    raise RuntimeError(f"hit (lane {lane}, key {n}) failed its recheck")
                status = ST_FOUND
        except Exception as e:  # reported to every rank below
            status, err = ST_ERROR, e
        records = exchange(dist, status, lane, n, device)
        failed = [r for r, rec in enumerate(records) if rec[0] == ST_ERROR]
        if failed:
            if err is not None:
                raise err
            raise RuntimeError(f"rank(s) {failed} failed; stopping")
        w = pick_winner(records)
        if w is not None:
            ident = share_identity(dist, ident if rank == w else None, w, device)
            return Winner(w, records[w][2], records[w][1], ident)
    return None


class GpuEngine:
    """One rank's GPU search: a Backend over seeded (or OS-random) walkers."""

    def __init__(self, device: int, prefix: str, aspect: str, seed: int | None, lanes: int = 0, iters: int = 4,
                 batch: int = 256):
        self.prefix, self.aspect = lx.prefix_parse(prefix), aspect
        self.b = lx.Backend(device=device, lanes=lanes, batch=batch)
        n = self.b.threads()
        if seed is not None:
            self.setup = lx.seeded_setup(seed, n)
        else:
            ed = lx.os_random(32)
            scal = np.stack([np.frombuffer(lx.random_start_scalar(), np.uint8) for _ in range(n)])
            self.setup = lx.WalkSetup(ed, lx.ed25519_public(ed), scal)
        self.b.init_from_scalars(self.setup.scalars)
        self.args = lx.make_launch_args(iters, self.setup.ed_pub, self.prefix, aspect=aspect)

    def launch(self) -> list[tuple[int, int]]:
        hits, _, _, _ = self.b.launch(self.args)
        return hits

    def identity(self, lane: int, n: int) -> bytes:
        return self.setup.identity(lane, n)

    def recheck(self, identity: bytes) -> bool:
        return lx.prefix_matches(self.prefix, lx.address_of_identity(identity, self.aspect))

    def close(self) -> None:
        self.b.close()


def main() -> int:
    import torch
    import torch.distributed as dist
    p = argparse.ArgumentParser(description="The search on every GPU of this node, one process per GPU.")
    p.add_argument("prefix")
    p.add_argument("--aspect", default=lx.ASPECT)
    p.add_argument("--seed", type=int, default=None)
    p.add_argument("--lanes", type=int, default=0)
    p.add_argument("--max-rounds", type=int, default=1 << 20)
    a = p.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    prefix = a.prefix.lower()
    path = f"{prefix}.identity"
    if rank == 0 and os.path.exists(path):
        print(f"{path} already exists; not overwriting it.", file=sys.stderr)
        return 1
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = f"cuda:{local}"
    seed = rank_seed(a.seed, rank) if a.seed is not None else None
    eng = GpuEngine(local, prefix, a.aspect, seed, lanes=a.lanes)
    try:
        w = replicated_search(dist if world > 1 else None, eng, a.max_rounds, dev)
    finally:
        eng.close()
        if world > 1:
            dist.destroy_process_group()
    if w is None:
        return 2
    if rank == 0:
        fd = os.open(path, os.O_WRONLY | os.O_CREAT | os.O_EXCL, 0o600)
        with os.fdopen(fd, "wb") as f:
            f.write(w.identity)
        print(f"Found {lx.address_of_identity(w.identity, a.aspect).hex()} on rank {w.rank}. Saved to {path}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
