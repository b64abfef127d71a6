"""Many searches at once on one B200: the search pool, the batched runner,
the autotuner and the serving loop.

The reference runs one search per process (GpuSearch, src/gpu/mod.rs:86-174);
to search for many prefixes it starts many processes.  Here:

- `Pool` wraps the C ABI's lxmfv_pool_*: a device-resident pool of walker
  lanes in which searches (each with its own prefix, aspect and identity) are
  admitted, walked together by one persistent kernel that takes 32-lane
  chunks from a device work queue, and retired;
- `run_batched` walks a fixed set of searches for a number of steps (the
  batched workload) and rechecks every hit on the CPU;
- `autotune` picks the pool's group size and step length for a workload by
  measuring them;
- `serve` is a request loop: searches arrive (a Poisson stream), are admitted
  while the pool has lanes for them (the memory budget), and are retired on
  their first hit, which frees lanes for the next ones while the others keep
  walking (continuous batching).  It reports wall-clock time-to-hit
  percentiles normalised by each search's expected time at its measured
  rate, beside the same in keys walked.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

import lxmfv as lx

BYTES_PER_LANE = 108  # lane state 64 + walk index 8 + submission staging 36 (lxmfv_pool_open)


@dataclass
class SearchSpec:
    """One search: prefix, aspect, identity (Ed25519 seed) and its lanes' start scalars."""
    prefix: str
    aspect: str
    ed_seed: bytes
    scalars: np.ndarray = field(repr=False)  # (lanes, 32) uint8, clamped

    @property
    def lanes(self) -> int:
        return self.scalars.shape[0]

    @property
    def nibbles(self) -> int:
        return len(self.prefix)

    @property
    def ed_pub(self) -> bytes:
        return lx.ed25519_public(self.ed_seed)

    def desc(self) -> lx.SearchDesc:
        d = lx.SearchDesc()
        d.ed[:] = lx.be_words(self.ed_pub)
        d.name_hash[:] = lx.name_hash_words(lx.name_hash(self.aspect))
        w, m = lx.prefix_words(lx.prefix_parse(self.prefix))
        d.want[:] = w
        d.mask[:] = m
        d.lanes = self.lanes
        return d

    def identity(self, lane: int, n: int) -> bytes:
        """The 64-byte identity of a hit (mod.rs:139-144)."""
        return lx.step_scalar(bytes(self.scalars[lane]), n) + self.ed_seed

    def recheck(self, lane: int, n: int) -> bool:
        """The reference's recheck (mod.rs:156-160): from scratch on the CPU."""
        return lx.prefix_matches(lx.prefix_parse(self.prefix), lx.address_of_identity(self.identity(lane, n), self.aspect))

    @classmethod
    def seeded(cls, seed: int, prefix: str, aspect: str = lx.ASPECT, lanes: int = 1024) -> "SearchSpec":
        """The seeding convention: identity and lane scalars from ChaCha20 stream `seed`."""
        ident, off = lx.seeded_identity(seed)
        scal = np.zeros((lanes, 32), np.uint8)
        scal[0] = np.frombuffer(ident[:32], np.uint8)
        if lanes > 1:
            scal[1:], _ = lx.seeded_scalars(seed, off, lanes - 1)
        return cls(prefix.lower(), aspect, ident[32:], scal)


class Pool:
    """The C ABI's search pool (lxmfv_pool_*)."""

    def __init__(self, device: int = 0, capacity_lanes: int = 0, memory_budget: int = 0, batch: int = 1024,
                 max_searches: int = 4096, max_hits: int = 65536, stream: int | None = None):
        L = lx.lib()
        o = lx.PoolOptions(device, capacity_lanes, memory_budget, batch, max_searches, max_hits, stream)
        h = C.c_void_p()
        rc = L.lxmfv_pool_open(C.byref(o), C.byref(h))
        self._h = h
        if rc != lx.OK:
            msg = L.lxmfv_pool_last_error(h).decode() if h.value else "pool open failed"
            L.lxmfv_pool_close(h)
            self._h = None
            raise lx.LxmfvError(rc, msg)
        self.batch = batch
        self.max_hits = max_hits
        self.specs: dict[int, SearchSpec] = {}

    def _check(self, rc: int) -> None:
        if rc != lx.OK:
            raise lx.LxmfvError(rc, lx.lib().lxmfv_pool_last_error(self._h).decode())

    def close(self) -> None:
        if self._h is not None:
            lx.lib().lxmfv_pool_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        i = lx.PoolInfo()
        self._check(lx.lib().lxmfv_pool_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in lx.PoolInfo._fields_}

    def submit(self, spec: SearchSpec) -> int:
        """Admits a search; raises LxmfvError (ERR_OVERFLOW) when it does not fit."""
        sid = C.c_uint32()
        scal = np.ascontiguousarray(spec.scalars, np.uint8)
        self._check(lx.lib().lxmfv_pool_submit(self._h, C.byref(spec.desc()), scal.ctypes.data_as(C.POINTER(C.c_uint8)),
                                               C.byref(sid)))
        self.specs[sid.value] = spec
        return sid.value

    def submit_many(self, specs: list[SearchSpec]) -> list[int]:
        """Admits the longest prefix of `specs` that fits (lxmfv_pool_submit_many:
        one start kernel for all, no wait); returns their ids.  Raises
        LxmfvError (ERR_OVERFLOW) when the first does not fit."""
        if not specs:
            return []
        descs = (lx.SearchDesc * len(specs))(*[sp.desc() for sp in specs])
        scal = np.ascontiguousarray(np.concatenate([sp.scalars for sp in specs]), np.uint8)
        ids = (C.c_uint32 * len(specs))()
        got = C.c_uint32()
        self._check(lx.lib().lxmfv_pool_submit_many(self._h, descs, len(specs),
                                                    scal.ctypes.data_as(C.POINTER(C.c_uint8)), ids, C.byref(got)))
        out = [ids[i] for i in range(got.value)]
        for sid, sp in zip(out, specs):
            self.specs[sid] = sp
        return out

    def retire(self, sid: int) -> None:
        self._check(lx.lib().lxmfv_pool_retire(self._h, sid))
        self.specs.pop(sid, None)

    def step(self, groups: int = 1) -> None:
        self._check(lx.lib().lxmfv_pool_step(self._h, groups))

    def poll(self, cap: int | None = None) -> tuple[list[tuple[int, int, int]], int]:
        cap = self.max_hits if cap is None else cap
        hits = (lx.PoolHit * max(cap, 1))()
        n = C.c_uint32()
        self._check(lx.lib().lxmfv_pool_poll(self._h, hits, cap, C.byref(n)))
        got = min(n.value, cap)
        return [(hits[i].search, hits[i].lane, hits[i].n) for i in range(got)], n.value

    def keys_per_lane(self, sid: int) -> int:
        return lx.lib().lxmfv_pool_keys_per_lane(self._h, sid)

    def last_step_ms(self) -> float:
        return lx.lib().lxmfv_pool_last_step_ms(self._h)


# ---- the batched workload

ASPECTS = ("lxmf.delivery", "nomadnetwork.node", "lxmf.propagation")


def batched_specs(n: int, seed: int, lanes: int, min_nibbles: int = 4, max_nibbles: int = 10) -> list[SearchSpec]:
    """n searches: prefix length uniform over [min, max] nibbles with random hex,
    aspects uniform over three, each with its own seeded identity (seed + i)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        nib = int(rng.integers(min_nibbles, max_nibbles + 1))
        prefix = "".join("0123456789abcdef"[x] for x in rng.integers(0, 16, nib))
        aspect = ASPECTS[int(rng.integers(0, len(ASPECTS)))]
        specs.append(SearchSpec.seeded(seed * 100003 + i, prefix, aspect, lanes))
    return specs


def run_batched(pool: Pool, specs: list[SearchSpec], steps: int, groups: int, warmup: int = 1,
                recheck_limit: int | None = None) -> dict:
    """Walks every search for `warmup` + `steps` steps, device-timing the
    steps; every hit of the timed steps is rechecked from scratch on the CPU
    (with recheck_limit, only each search's first that many: the autotuner's
    quick sweeps)."""
    sids = [pool.submit(s) for s in specs]
    for _ in range(warmup):
        pool.step(groups)
    pool.poll()
    lanes = sum(s.lanes for s in specs)
    ms = 0.0
    hits_all: list[tuple[int, int, int]] = []
    total_hits = 0
    for _ in range(steps):
        pool.step(groups)
        h, n = pool.poll()
        ms += pool.last_step_ms()
        hits_all += h
        total_hits += n
    per_search: dict[int, int] = {}
    bad = 0
    checked = 0
    for sid, lane, n in hits_all:
        c = per_search.get(sid, 0)
        if recheck_limit is None or c < recheck_limit:
            checked += 1
            bad += 0 if pool.specs[sid].recheck(lane, n) else 1
        per_search[sid] = c + 1
    keys = lanes * pool.batch * groups * steps
    for sid in sids:
        pool.retire(sid)
    return {"keys_per_s": keys / (ms * 1e-3), "keys": keys, "ms": ms, "searches": len(specs), "lanes": lanes,
            "hits": total_hits, "hits_rechecked": checked, "rechecked_bad": bad, "groups_per_step": groups,
            "batch": pool.batch}


def autotune(device: int, specs_fn, lanes_total: int, batches=(64, 128, 256, 512, 1024), groups=(1, 2, 4),
             steps: int = 3) -> dict:
    """Measures the pool's aggregate keys/s for each keys-per-group and step
    length on the given search mix; returns the fastest with all results."""
    results = []
    for b in batches:
        with Pool(device=device, capacity_lanes=lanes_total, batch=b) as pool:
            for g in groups:
                r = run_batched(pool, specs_fn(), steps=steps, groups=g, warmup=1, recheck_limit=2)
                results.append({"batch": b, "groups": g, "keys_per_s": r["keys_per_s"], "bad": r["rechecked_bad"]})
    best = max(results, key=lambda r: r["keys_per_s"])
    return {"best": best, "results": results}


# ---- the serving loop

@dataclass
class Request:
    arrival: float     # seconds from the start
    spec: SearchSpec
    admitted: float | None = None
    done: float | None = None
    tries: int | None = None   # keys before and including the hit, in walk order
    walked: int | None = None  # keys the search had walked when its hit was reported
    hit: tuple[int, int] | None = None  # (lane, n)
    failed: bool = False  # its hit failed the recheck: no identity is returned


def lanes_by_difficulty(nibbles: int, base: int = 64, cap: int = 32768) -> int:
    """Lanes for a request: 64 for 5 nibbles, 16 times more per further nibble,
    at most `cap`, so that expected steps to a hit stay about level."""
    return int(min(cap, max(32, base * 16 ** max(0, nibbles - 5))))


def poisson_requests(rate: float, duration: float, seed: int, lanes, min_nibbles: int = 5,
                     max_nibbles: int = 9, p: float = 0.9) -> list[Request]:
    """Arrivals of a Poisson stream; prefix length min + Geometric(p) - 1,
    redrawn above max (a truncated geometric); random hex; aspects uniform over
    three; seeded identities.  `lanes` is a count or a function of nibbles."""
    rng = np.random.default_rng(seed)
    lanes_of = lanes if callable(lanes) else (lambda _n, k=lanes: k)
    t, reqs = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        while True:
            nib = min_nibbles + int(rng.geometric(p)) - 1
            if nib <= max_nibbles:
                break
        prefix = "".join("0123456789abcdef"[x] for x in rng.integers(0, 16, nib))
        aspect = ASPECTS[int(rng.integers(0, len(ASPECTS)))]
        reqs.append(Request(t, SearchSpec.seeded(seed * 1000003 + len(reqs), prefix, aspect, lanes_of(nib))))
    return reqs


def expected_tries(nibbles: int) -> float:
    return 16.0 ** nibbles


def serve(pool: Pool, requests: list[Request], groups: int = 1, time_limit: float | None = None) -> dict:
    """Runs the request loop until every request is done (or time_limit).
    Each step: admit arrived requests while the pool has lanes (continuous
    batching), walk every admitted search one step, retire searches on their
    first hit (the hit with the smallest (n, lane), rechecked from scratch).
    A hit that fails its recheck fails its request (the reference stops with
    an error, main.rs:310-313): the search is retired without an identity and
    counted in `rechecked_bad`; the other requests go on.  A request that an
    empty pool refuses (larger than its memory budget) fails at once."""
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    waiting: deque[Request] = deque()
    active: dict[int, Request] = {}
    done: list[Request] = []
    failed: list[Request] = []
    t0 = time.perf_counter()
    steps = 0
    keys = 0
    busy_ms = 0.0
    step_wall = 0.0  # wall time of the loop's step + poll calls
    bad = 0
    while pending or waiting or active:
        now = time.perf_counter() - t0
        if time_limit is not None and now > time_limit:
            break
        while pending and pending[0].arrival <= now:
            waiting.append(pending.popleft())
        while waiting:
            # Everything that arrived and fits, in arrival order, in one
            # admission (one start kernel, queued ahead of the next step).
            try:
                sids = pool.submit_many([r.spec for r in waiting])
            except lx.LxmfvError as e:
                if e.code != lx.ERR_OVERFLOW:
                    raise
                if active:
                    break  # no lanes free: it waits for a retirement
                # Refused by an empty pool: larger than the whole memory budget.
                r = waiting.popleft()
                r.failed = True
                r.done = time.perf_counter() - t0
                failed.append(r)
                continue
            t_adm = time.perf_counter() - t0
            for sid in sids:
                r = waiting.popleft()
                r.admitted = t_adm
                active[sid] = r
            if waiting and active:
                break  # the rest wait for lanes
        if not active:
            if pending:
                time.sleep(max(0.0, min(pending[0].arrival - now, 0.05)))
            continue
        lanes = sum(r.spec.lanes for r in active.values())
        t_step = time.perf_counter()
        pool.step(groups)
        hits, _ = pool.poll()
        steps += 1
        keys += lanes * pool.batch * groups
        busy_ms += pool.last_step_ms()
        step_wall += time.perf_counter() - t_step
        t_now = time.perf_counter() - t0
        first: dict[int, tuple[int, int]] = {}
        for sid, lane, n in hits:
            if sid in active and (sid not in first or (n, lane) < (first[sid][1], first[sid][0])):
                first[sid] = (lane, n)
        for sid, (lane, n) in first.items():
            r = active.pop(sid)
            if not r.spec.recheck(lane, n):
                bad += 1
                r.failed = True
                r.done = t_now
                pool.retire(sid)
                failed.append(r)
                continue
            r.done = t_now
            r.hit = (lane, n)
            # Lanes advance in step: the hit is key number n * lanes + lane + 1 in walk order.
            r.tries = n * r.spec.lanes + lane + 1
            r.walked = pool.keys_per_lane(sid) * r.spec.lanes
            pool.retire(sid)
            done.append(r)
    wall = time.perf_counter() - t0
    lane_rate = steps * pool.batch * groups / step_wall if step_wall > 0 else 0.0
    return summarise(done, requests, wall, keys, busy_ms, steps, bad, failed=len(failed), lane_rate=lane_rate)


def wall_time_to_hit(r: Request) -> float:
    """A done request's wall-clock time to hit over its expected time at its
    measured rate.  The time to hit runs from arrival (so it includes the
    queue wait) to the poll that reported the hit (so it includes the rest of
    that step).  The rate is the request's own: the keys it walked over its
    wall time in the pool, arrival excluded, so a loaded pool's slower steps
    are in the rate and the wait is in the time.  The expected time is then
    16^L over that rate, and an exponential time to hit has the quantiles
    ln 2, ln 20 and ln 100 at p50, p95 and p99."""
    in_pool = r.done - r.admitted
    if in_pool <= 0 or not r.walked:
        return float("nan")
    expected_s = expected_tries(r.spec.nibbles) * in_pool / r.walked
    return (r.done - r.arrival) / expected_s


def summarise(done: list[Request], requests: list[Request], wall: float, keys: int, busy_ms: float, steps: int,
              bad: int, failed: int = 0, lane_rate: float = 0.0) -> dict:
    norm_tries = np.array([r.tries / expected_tries(r.spec.nibbles) for r in done]) if done else np.zeros(0)
    # Time in service at the search's own (constant, per step) key rate is its
    # walked keys over that rate, so its time over the expected time is the
    # walked keys over the expected tries: the tries, rounded up to the end of
    # the step that reported the hit.
    norm_service = np.array([r.walked / expected_tries(r.spec.nibbles) for r in done]) if done else np.zeros(0)
    # Wall clock: arrival to the reported hit, over 16^L at the request's own
    # measured rate (wall_time_to_hit), and over 16^L at the pool's mean rate
    # per lane (every step's keys per lane over the wall time of the steps)
    # times the request's lanes.
    norm_wall = np.array([wall_time_to_hit(r) for r in done]) if done else np.zeros(0)
    norm_wall_pool = (np.array([(r.done - r.arrival) * r.spec.lanes * lane_rate / expected_tries(r.spec.nibbles)
                                for r in done]) if done and lane_rate > 0 else np.zeros(0))
    rate = keys / (busy_ms * 1e-3) if busy_ms > 0 else 0.0
    q = lambda a, p: float(np.quantile(a, p)) if len(a) else float("nan")  # noqa: E731
    targets = {"p50": math.log(2), "p95": math.log(20), "p99": math.log(100)}
    pct = (("p50", .5), ("p95", .95), ("p99", .99))
    wall_q = {k: q(norm_wall, p) for k, p in pct}
    out = {
        "requests": len(requests), "done": len(done), "failed": failed, "wall_s": wall, "steps": steps,
        "aggregate_keys_per_s": rate, "busy_fraction": busy_ms * 1e-3 / wall if wall > 0 else 0.0,
        "rechecked_bad": bad,
        "time_to_hit_over_expected": wall_q,
        "time_to_hit_deviation": {k: wall_q[k] / targets[k] - 1 for k in wall_q},
        "time_to_hit_at_pool_rate": {k: q(norm_wall_pool, p) for k, p in pct},
        "lane_keys_per_s": lane_rate,
        "tries_over_expected": {k: q(norm_tries, p) for k, p in pct},
        "service_time_over_expected": {k: q(norm_service, p) for k, p in pct},
        "targets": targets,
        "latency_s": {k: q(np.array([r.done - r.arrival for r in done]), p) for k, p in (("p50", .5), ("p95", .95), ("p99", .99))},
        "queue_wait_s": {k: q(np.array([r.admitted - r.arrival for r in done]), p) for k, p in (("p50", .5), ("p99", .99))},
    }
    return out
