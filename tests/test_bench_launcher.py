"""bench.py's own launcher and its multi-rank plumbing, on the CPU: with
--gpus 2 and no launcher around it, bench.py starts two ranks under
torch.distributed.run; the ranks walk disjoint seeded walkers (seed +
1000 * rank), the slowest rank's time sets the whole-job rate, and rank 0
alone prints one JSON line with n_gpus 2.  A world size that does not match
--gpus is refused.  The engine is tests/bench_stub.py (the library's CPU
walk over gloo); the GPU engine runs the same code around the CUDA kernels."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _env(**kw):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                             "MASTER_PORT")}
    env.update(kw)
    return env


def _bench(args, env):
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=300)


def test_gpus_2_starts_two_ranks_and_prints_one_line(oracle):
    from tests import bench_stub

    p = _bench(["--gpus", "2", "--steps", "2", "--warmup", "3", "--lanes", "3",
                "--engine", "tests.bench_stub:measure"], _env())
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["scaling"] == "weak"
    ranks = line["ranks"]
    assert [r["rank"] for r in ranks] == [0, 1]
    assert [r["seed"] for r in ranks] == [3, 1003]  # seed + 1000 * rank: disjoint walkers
    keys = 3 * bench_stub.KEYS * 2
    assert line["value"] == pytest.approx(2 * keys / (max(r["ms"] for r in ranks) * 1e-3), rel=1e-9)
    # Each rank's hits are its own walkers', as the oracle's search finds them.
    nh = oracle.name_hash("lxmf.delivery")
    pfx = oracle.prefix_parse(line["prefix"][:bench_stub.NIBBLES])
    first = 3 * bench_stub.KEYS
    for r in ranks:
        k0, ed_seed, off = oracle.seeded_identity(r["seed"])
        starts = [k0] + [bytes(s) for s in oracle.seeded_scalars(r["seed"], off, 2)[0]]
        expect = set()
        for lane, st in enumerate(starts):
            h, _ = oracle.search_window(st, oracle.ed25519_public(ed_seed), nh, pfx, first + keys // 3)
            expect.update((lane, int(n)) for n in h if n >= first)
        assert {tuple(h) for h in r["hits"]} == expect
    assert ranks[0]["hits"] != ranks[1]["hits"]


def test_a_world_size_other_than_gpus_is_refused():
    p = _bench(["--gpus", "2", "--steps", "1", "--warmup", "3", "--engine", "tests.bench_stub:measure"],
               _env(WORLD_SIZE="1", RANK="0", LOCAL_RANK="0"))
    assert p.returncode != 0 and "does not match" in p.stderr


def test_every_default_section_has_its_ncu_counts():
    """The bench's roofline for each default plain-search section (the headline
    G, and B = 64 for both walks) comes from per-key ncu counts: ALU-pipe and
    IMAD-class instructions, all instructions and DRAM bytes."""
    sys.path.insert(0, ROOT)
    import bench

    for key in (("group", bench.BATCH), ("group", 64), ("xadd", 64)):
        counts = bench.NCU_PER_KEY[key]
        assert {"alu", "imad", "inst", "dram_bytes"} <= set(counts), key
        assert counts["alu"] + counts["imad"] < counts["inst"]
    # The algorithmic field work per key falls as the group grows (one inversion per G keys).
    assert bench.wide_products_per_key("group", 1024) < bench.wide_products_per_key("group", 64)
    assert bench.wide_products_per_key("group", 64) < bench.wide_products_per_key("xadd", 64)


def test_reference_arm_under_two_ranks_prints_one_line():
    """`bench.py --impl reference --gpus 2`, as the scaling run launches it:
    rank 0 alone times the reference's CPU walk and prints one line with
    impl "reference"; the other rank exits 0 without work."""
    p = _bench(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"], _env())
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, p.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
