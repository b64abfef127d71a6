"""A host-side engine for bench.py's multi-rank plumbing, for
tests/test_bench_launcher.py: `python bench.py --gpus 2 --engine
tests.bench_stub:measure` runs two ranks over gloo on the CPU.

Each rank walks its seeded walkers (lane 0 the seed's identity scalar, lane t
the t-th further draw, as on the GPU) with the library's CPU walk and
address chain (lxmfv_cpu_walk, lxmfv_cpu_addresses), KEYS keys per lane per
step, and reports the hits of the bench prefix's first two nibbles, so that
the test can check them against the oracle."""
import time

import numpy as np

import lxmfv as lx

KEYS = 128  # keys per lane per step
NIBBLES = 2  # prefix digits searched (the bench's 8 would find nothing here)


def measure(seed: int, steps: int, warmup: int, prefix: str, lanes: int) -> dict:
    setup = lx.seeded_setup(seed, lanes)
    ed = np.frombuffer(setup.ed_pub, np.uint8)
    pfx = lx.prefix_parse(prefix[:NIBBLES])
    pos = 0

    def step() -> list[tuple[int, int]]:
        nonlocal pos
        hits = []
        for lane, k in enumerate(setup.scalars):
            keys = lx.cpu_walk(lx.step_scalar(bytes(k), pos), KEYS)
            addrs = lx.cpu_addresses(np.concatenate([keys, np.tile(ed, (KEYS, 1))], 1))
            hits += [(lane, pos + i) for i in range(KEYS) if lx.prefix_matches(pfx, bytes(addrs[i]))]
        pos += KEYS
        return hits

    for _ in range(warmup):
        step()
    first = pos
    t0 = time.perf_counter()
    hits = []
    for _ in range(steps):
        hits += step()
    ms = (time.perf_counter() - t0) * 1e3
    return {"keys_per_step": lanes * KEYS, "ms": ms, "hits": hits, "first_key": first}
