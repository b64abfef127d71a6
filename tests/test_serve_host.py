"""The serving loop (lxmfv_serve.serve) on the host, with failures injected
there and no GPU: a pool stand-in whose hits come from the oracle's walk, one
search made to report a corrupted hit, admission against a small memory
budget, and a request larger than the whole budget."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "lxmf-vanity_b200"))
sys.path.insert(0, os.path.join(os.path.dirname(__file__), ".."))

import lxmfv as lx  # noqa: E402
import lxmfv_serve as srv  # noqa: E402
from oracle import oracle as O  # noqa: E402


class HostPool:
    """lxmfv_serve.Pool's interface on the host.  Every search has one lane;
    its first hit is the oracle's first match on that lane's walk, reported
    once the search has walked past it.  Searches admitted in the positions
    listed in `corrupt` report the key after their hit instead."""

    def __init__(self, capacity_lanes: int, batch: int = 64, corrupt=()):
        self.capacity, self.batch, self.corrupt = capacity_lanes, batch, set(corrupt)
        self.used = self.admitted = self.max_active = 0
        self.active, self.walked, self.first, self.retired = {}, {}, {}, []

    def submit(self, spec: srv.SearchSpec) -> int:
        if self.used + spec.lanes > self.capacity:
            raise lx.LxmfvError(lx.ERR_OVERFLOW, "no lanes free")
        sid = self.admitted
        self.admitted += 1
        self.used += spec.lanes
        self.active[sid], self.walked[sid] = spec, 0
        hits, _ = O.search_window(bytes(spec.scalars[0]), O.ed25519_public(spec.ed_seed), O.name_hash(spec.aspect),
                                  O.prefix_parse(spec.prefix), 1 << 14)
        assert len(hits), "the oracle window holds a hit"
        self.first[sid] = int(hits[0]) + (1 if sid in self.corrupt else 0)
        self.max_active = max(self.max_active, len(self.active))
        return sid

    def submit_many(self, specs: list) -> list:
        """lxmfv_pool_submit_many: the longest prefix that fits; overflow when the first does not."""
        ids = []
        for spec in specs:
            if self.used + spec.lanes > self.capacity:
                break
            ids.append(self.submit(spec))
        if not ids:
            raise lx.LxmfvError(lx.ERR_OVERFLOW, "no lanes free")
        return ids

    def step(self, groups: int = 1) -> None:
        for sid in self.active:
            self.walked[sid] += self.batch * groups

    def poll(self):
        hits = [(sid, 0, self.first[sid]) for sid in self.active if self.first[sid] < self.walked[sid]]
        return hits, len(hits)

    def keys_per_lane(self, sid: int) -> int:
        return self.walked[sid]

    def last_step_ms(self) -> float:
        return 1.0

    def retire(self, sid: int) -> None:
        self.used -= self.active.pop(sid).lanes
        self.retired.append(sid)


def requests(n: int, lanes: int = 1) -> list:
    return [srv.Request(arrival=0.0, spec=srv.SearchSpec.seeded(40 + i, ["c3", "5a", "e0", "b1"][i % 4],
                                                                srv.ASPECTS[i % 3], lanes=lanes))
            for i in range(n)]


def test_a_corrupted_hit_fails_only_its_request():
    reqs = requests(4)
    pool = HostPool(capacity_lanes=4, corrupt={1})
    out = srv.serve(pool, reqs, time_limit=60)
    assert out["rechecked_bad"] == 1 and out["failed"] == 1 and out["done"] == 3
    assert reqs[1].failed and reqs[1].hit is None
    for r in reqs[:1] + reqs[2:]:
        assert not r.failed and r.spec.recheck(*r.hit)
        assert lx.prefix_matches(lx.prefix_parse(r.spec.prefix),
                                 lx.address_of_identity(r.spec.identity(*r.hit), r.spec.aspect))
    assert sorted(pool.retired) == [0, 1, 2, 3] and pool.used == 0


def test_admission_waits_for_lanes():
    reqs = requests(6)
    pool = HostPool(capacity_lanes=2)
    out = srv.serve(pool, reqs, time_limit=60)
    assert out["done"] == 6 and out["failed"] == 0 and out["rechecked_bad"] == 0
    assert pool.max_active == 2 and pool.used == 0
    # Searches admitted later waited for a retirement.
    assert max(r.admitted for r in reqs) >= min(r.done for r in reqs)


def test_a_request_larger_than_the_pool_fails_at_once():
    reqs = requests(3)
    reqs[1] = srv.Request(arrival=0.0, spec=srv.SearchSpec.seeded(7, "c3", lanes=8))
    pool = HostPool(capacity_lanes=2)
    out = srv.serve(pool, reqs, time_limit=60)
    assert reqs[1].failed and out["failed"] == 1 and out["done"] == 2
    assert out["rechecked_bad"] == 0


def test_wall_clock_time_to_hit_is_normalised_by_the_requests_own_rate():
    """wall_time_to_hit: (done - arrival) over 16^L at the request's rate in
    the pool (keys walked over done - admitted); the queue wait raises it, a
    slower pool does not."""
    spec = srv.SearchSpec.seeded(5, "abcde", lanes=32)  # 5 nibbles: 16^5 expected tries
    expected = 16.0 ** 5
    fast = srv.Request(arrival=0.0, spec=spec, admitted=0.0, done=1.0, walked=int(expected), tries=int(expected))
    slow = srv.Request(arrival=0.0, spec=spec, admitted=0.0, done=2.0, walked=int(expected), tries=int(expected))
    waited = srv.Request(arrival=0.0, spec=spec, admitted=1.0, done=2.0, walked=int(expected), tries=int(expected))
    assert srv.wall_time_to_hit(fast) == pytest.approx(1.0)
    assert srv.wall_time_to_hit(slow) == pytest.approx(1.0)   # the same keys at half the rate
    assert srv.wall_time_to_hit(waited) == pytest.approx(2.0)  # a second of queue wait before a second in the pool
    out = srv.summarise([fast, slow, waited], [fast, slow, waited], wall=2.0, keys=3 * int(expected), busy_ms=2000.0,
                        steps=3, bad=0, lane_rate=expected / 32)
    assert out["time_to_hit_over_expected"]["p50"] == pytest.approx(1.0)
    assert out["time_to_hit_at_pool_rate"]["p50"] == pytest.approx(2.0)  # 2 s at the pool's mean rate of 1 per s
