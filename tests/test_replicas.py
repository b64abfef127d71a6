"""The replicated (multi-GPU) search's host logic with world_size 2 over gloo,
on the CPU: disjoint seeded walkers per rank, one common winner (the smallest
(n, lane, rank), checked against the oracle's search over every rank's
walkers), max-over-ranks timing, and a failing rank that stops every rank
with an error instead of leaving it waiting in a collective."""
import json
import os
import socket
import subprocess
import sys

import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WORKER = os.path.join(ROOT, "tests", "replica_worker.py")
sys.path.insert(0, os.path.join(ROOT, "lxmf-vanity_b200"))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(case: str, world: int = 2, **kw) -> list[dict]:
    port = _free_port()
    extra = [f"--{k}={v}" for k, v in kw.items()]
    procs = [subprocess.Popen([sys.executable, WORKER, "--rank", str(r), "--world", str(world), "--port", str(port),
                               "--case", case] + extra, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                              env=dict(os.environ, MASTER_ADDR="127.0.0.1"))
             for r in range(world)]
    outs = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail(f"rank timed out in case {case}")
        assert p.returncode == 0, se[-2000:]
        outs.append(json.loads(so.strip().splitlines()[-1]))
    return sorted(outs, key=lambda o: o["rank"])


def _oracle_winner(seed: int, world: int, prefix: str, aspect: str, lanes: int = 4, keys_per_round: int = 256):
    """The first (round, n, lane, rank) hit over all ranks' seeded walkers."""
    import lxmfv_replicas as rep
    best = None
    for r in range(world):
        k0, ed_seed, off = O.seeded_identity(rep.rank_seed(seed, r))
        starts = [k0] + [bytes(s) for s in O.seeded_scalars(rep.rank_seed(seed, r), off, lanes - 1)[0]]
        for lane, st in enumerate(starts):
            hits, _ = O.search_window(st, O.ed25519_public(ed_seed), O.name_hash(aspect), O.prefix_parse(prefix),
                                      keys_per_round * 64)
            if len(hits):
                n = int(hits[0])
                cand = (n // keys_per_round, n, lane, r, O.step_scalar(st, n) + ed_seed)
                best = cand if best is None or cand[:4] < best[:4] else best
    return best


@pytest.mark.parametrize("seed,prefix,aspect", [(5, "abc", "lxmf.delivery"), (12, "d0d", "nomadnetwork.node")])
def test_ranks_agree_on_the_oracle_winner(seed, prefix, aspect):
    outs = _run("search", seed=seed, prefix=prefix, aspect=aspect)
    winners = [o["winner"] for o in outs]
    assert winners[0] is not None and all(w == winners[0] for w in winners)
    rnd, n, lane, rank, ident = _oracle_winner(seed, 2, prefix, aspect)
    w = winners[0]
    assert (w["rank"], w["lane"], w["n"]) == (rank, lane, n)
    assert bytes.fromhex(w["identity"]) == ident
    assert O.prefix_matches(O.prefix_parse(prefix), O.address_of_identity(ident, aspect))
    # Every rank stopped in the same round: the winner's.
    assert all(o["launches"] == rnd + 1 for o in outs)


def test_rank_seeds_are_disjoint():
    import lxmfv_replicas as rep
    seen = set()
    for r in range(8):
        k0, _, off = O.seeded_identity(rep.rank_seed(3, r))
        for s in [k0] + [bytes(x) for x in O.seeded_scalars(rep.rank_seed(3, r), off, 63)[0]]:
            assert s not in seen
            seen.add(s)


def test_max_over_ranks_and_the_aggregate_rate():
    outs = _run("max")
    assert [o["max"] for o in outs] == [2.5, 2.5]
    assert all(o["rate"] == pytest.approx(2 * 1000.0 / 2.5) for o in outs)


def test_a_failing_rank_stops_every_rank():
    outs = _run("fail", prefix="0123456789")  # no hit in 64 rounds: only the failure ends it
    assert all("error" in o for o in outs), outs
    assert "injected engine failure" in outs[1]["error"]
    assert "rank(s) [1] failed" in outs[0]["error"]
    assert all(o["launches"] == 2 for o in outs)


@pytest.mark.gpu
def test_gpu_engine_single_rank_finds_the_plain_search_hit():
    """World size 1 on the GPU: the replicated search's winner is the plain
    search's first hit (smallest (n, lane)) over the same seeded walkers."""
    import lxmfv as lx
    import lxmfv_replicas as rep
    eng = rep.GpuEngine(0, "b00b", "lxmf.delivery", seed=rep.rank_seed(4, 0), lanes=8192, iters=2, batch=256)
    try:
        w = rep.replicated_search(None, eng, max_rounds=64)
    finally:
        eng.close()
    assert w is not None and w.rank == 0
    # The same walkers through the plain Backend, launch by launch.
    setup = lx.seeded_setup(rep.rank_seed(4, 0), 8192)
    with lx.Backend(device=0, lanes=8192, batch=256) as b:
        b.init_from_scalars(setup.scalars)
        args = lx.make_launch_args(2, setup.ed_pub, lx.prefix_parse("b00b"))
        for _ in range(64):
            hits, _, _, _ = b.launch(args)
            if hits:
                lane, n = min(hits, key=lambda h: (h[1], h[0]))
                break
    assert (w.lane, w.n) == (lane, n)
    assert w.identity == setup.identity(lane, n)
    assert O.prefix_matches(O.prefix_parse("b00b"), O.address_of_identity(w.identity))
