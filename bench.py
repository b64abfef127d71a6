#!/usr/bin/env python3
"""Benchmark of the B200 key-walk search: keys/s on the plain GPU search.

Workload (the plain GPU search): one 8-hex-digit prefix (numpy-seeded),
aspect lxmf.delivery, every lane starting from its own seeded clamped X25519
scalar (ChaCha20 stream of the seed) with one shared Ed25519 key, 2^36 keys
walked in total over the timed steps (a step is one launch that walks every
lane `iters` groups further).  Keys per inversion: the tuned 1024 for the
headline; the same 2^36 keys again at 64 (the reference kernel's BATCH), with
the grouped walk (`at_batch_64`) and with the x-only walk, the reference's
algorithm (`xadd_b64`).  Synthetic, seeded inputs; no dataset is involved.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 and no launcher around it, bench.py starts its N ranks
itself under torch.distributed.run (one process per GPU); under a launcher
the world size must equal N.  Prints one JSON line on rank 0.  `value` is
device-timed (CUDA events on the launching stream, max over ranks), `e2e`
goes through the C ABI's synchronous lxmfv_launch with host buffers,
`cpu_baseline` is the restated CPU search on this host's cores, `roofline`
relates the walk kernel's ALU-pipe work (ncu counts per key) to the measured
ALU rate of this GPU (and `roofline.imad_ncu` its IMAD-class instructions to
the measured IMAD rate), `reference_cuda_kernel` times the reference's own
CUDA kernel on this GPU and `cpu_search` this library's CPU search (the
reference's default mode).  With --impl reference, the reference's own
kernel body (src/gpu/common.h, built for the host) is timed on the host
cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "lxmf-vanity_b200"))

import lxmfv_replicas as replicas  # noqa: E402  (rank seeds, max over ranks)

TOTAL_KEYS = 1 << 36
BATCH = 1024
SEED = 3
METRIC = "keys/s, plain GPU search (one 8-hex prefix, seeded walkers, 2^36 keys), bit-exact"


def field_ops_per_key(walk: str, b: int) -> tuple[float, float]:
    """(multiplies, squarings) per key, counted from the kernels' code.
    x-only walk, B keys per inversion: 8B + 11 M and 2B + 254 S per batch.
    Grouped walk, G = 2m keys per group: (5m + 13) M and (2m + 255) S per group."""
    if walk == "xadd":
        return 8 + 11 / b, 2 + 254 / b
    m = b // 2
    return (5 * m + 13) / b, (2 * m + 255) / b


# Per key, from ncu captures of each kernel on a small case (profiles/walk_group_g1024_plain_search.md,
# profiles/walk_group_g64_plain_search.md, profiles/walk_xadd_b64_plain_search.md; the G = 512, 256 and x-only
# B = 128 rows from the earlier captures in profiles/):
#   alu: ALU-pipe lane operations (the binding pipe): sm__inst_executed_pipe_alu.sum x 32 / keys (earlier rows:
#        ALU pipe active % x 64 lanes x SMs x clock / keys per second);
#   imad: IMAD-class instructions per key: sm__inst_executed_pipe_fmaheavy.sum x 32 / keys, the pipe that
#        executes IMAD, IMAD.HI, IMAD.WIDE and IMAD.X (these kernels run no floating point);
#   inst: all instructions (smsp__inst_executed.sum x 32 / keys); dram_bytes: DRAM read + write.
NCU_PER_KEY = {
    ("group", 1024): {"alu": 3213, "imad": 2219, "inst": 5764, "dram_bytes": 32.0},
    ("group", 512): {"alu": 3243, "inst": 5823, "dram_bytes": 31.6},
    ("group", 256): {"alu": 3288, "inst": 5935, "dram_bytes": 31.1},
    ("group", 64): {"alu": 3546, "imad": 2678, "inst": 6605, "dram_bytes": 24.8},
    ("xadd", 128): {"alu": 4166, "inst": 8120, "dram_bytes": 131.9},
    ("xadd", 64): {"alu": 4319, "imad": 3740, "inst": 8562, "dram_bytes": 132.1},
}


def wide_products_per_key(walk: str, b: int) -> float:
    """32x32->64 products per key with 8 x 32-bit limbs: a field multiply is
    64 + 8 (the fold by 38), a square 36 + 8."""
    mul, sqr = field_ops_per_key(walk, b)
    return mul * 72 + sqr * 44


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--lanes", type=int, default=0, help="walker lanes per GPU (0: two full waves)")
    p.add_argument("--batch", type=int, default=BATCH, help="keys per inversion (grouped walk: 32..1024)")
    p.add_argument("--walk", choices=["group", "xadd"], default="group")
    p.add_argument("--block", type=int, default=0)
    p.add_argument("--total-keys", type=float, default=float(TOTAL_KEYS))
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-cpu-search", action="store_true", help="skip timing this library's CPU search")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's CUDA kernel")
    p.add_argument("--no-b64", action="store_true", help="skip the measurements at B = 64 (grouped and x-only walks)")
    p.add_argument("--engine", default="gpu",
                   help="gpu (the CUDA kernels, NCCL between ranks), or module:function, a host-side stand-in "
                        "measured over gloo that the launcher's tests use")
    p.add_argument("--no-batched", action="store_true", help="skip the 256-search batched measurement")
    p.add_argument("--served-seconds", type=float, default=60.0,
                   help="length of the served-requests run (0: skip); the full served workload is 600")
    return p.parse_args()


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "out", "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline_port(prefix: str, seconds: float = 2.5) -> dict:
    """The restated CPU search (KeyWalk + search of src/main.rs, B = 256,
    5 x 51-bit field) on every host core, for a bounded sample."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    pfx = O.prefix_parse(prefix)
    rate, keys, _ = O.bench_search(threads, 1 << 14, SEED, pfx)  # calibration
    per_thread = max(1 << 14, int(rate * seconds / threads))
    rate, keys, _ = O.bench_search(threads, per_thread, SEED, pfx)
    return {"value": rate, "unit": "keys/s", "cores": threads, "kind": "port",
            "sample": f"{keys} keys: {threads} threads x {per_thread} keys each from seeded starts, "
                      f"prefix {prefix}, restated KeyWalk (B=256) + double SHA-256 per key"}


def cpu_search_rate(seconds: float = 3.0) -> dict:
    """This library's own CPU search (lxmfv_cpu_search: the reference's
    default mode) on every host core for `seconds`, with a prefix it will not
    find in that time."""
    import threading

    import lxmfv as lx
    threads = os.cpu_count() or 1
    s = lx.CpuSearch(lx.prefix_parse("0123456789abcdef"), threads=threads, seed=SEED)
    timer = threading.Timer(seconds, s.stop)
    t0 = time.perf_counter()
    timer.start()
    found = s.run()
    dt = time.perf_counter() - t0
    return {"value": s.tries / dt, "unit": "keys/s", "threads": threads, "seconds": round(dt, 2),
            "found": found is not None,
            "api": "lxmfv_cpu_search (grouped affine walk, 5 x 51-bit field on 8 AVX-512 IFMA lanes where "
                   "present; SHA-256 16 keys at a time with AVX-512F, else the x86 SHA extensions, else portable C)"}


def reference_cpu(prefix: str, steps: int, warmup: int, step_seconds: float = 2.0) -> dict:
    """The reference's own kernel body (common.h walk_thread, B = 64) built for
    the host, on every host core.  Each step walks a bounded sample."""
    import ctypes as C

    import numpy as np

    from oracle import oracle as O
    r = O.ref()
    workers = os.cpu_count() or 1
    if r is None:
        port = cpu_baseline_port(prefix, step_seconds)
        return dict(port, steps=0)
    lanes = workers * 4
    ident = O.seeded_identity(SEED)
    k0, ed_seed, off = ident
    scal, _ = O.seeded_scalars(SEED, off, lanes - 1)
    starts = [k0] + [bytes(s) for s in scal]
    upc = np.zeros((lanes, 16), np.uint32)
    for t, k in enumerate(starts):
        upc[t, :8] = np.frombuffer(O.x25519_base(O.previous_scalar(k)), "<u4")
        upc[t, 8:] = np.frombuffer(O.x25519_base(k), "<u4")
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    state = np.zeros(lanes * 40, np.int32)
    ns = np.zeros(lanes, np.uint64)
    r.ref_init_walk(P(state, C.c_int32), P(upc, C.c_uint32), lanes)
    ed = np.frombuffer(O.ed25519_public(ed_seed), ">u4").astype(np.uint32)
    nh = O.name_hash("lxmf.delivery")
    nhw = [int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)]
    w, m = O.prefix_words(O.prefix_parse(prefix))
    want, mask = np.array(w, np.uint32), np.array(m, np.uint32)
    hc = np.zeros(1, np.uint32)
    hits = np.zeros(2 * 4096, np.uint64)
    q = np.frombuffer(O.u8b(), "<u4").astype(np.uint32)

    def run(iters: int) -> float:
        return r.ref_bench_walk(workers, P(state, C.c_int32), P(ns, C.c_uint64), lanes, iters, P(ed, C.c_uint32),
                                nhw[0], nhw[1], nhw[2], P(want, C.c_uint32), P(mask, C.c_uint32), P(hc, C.c_uint32),
                                P(hits, C.c_uint64), 4096, P(q, C.c_uint32))

    rate = run(1)
    iters = max(1, int(rate * step_seconds / (lanes * r.ref_batch())))
    for _ in range(warmup):
        run(iters)
    t0 = time.perf_counter()
    for _ in range(steps):
        run(iters)
    dt = time.perf_counter() - t0
    keys = steps * lanes * iters * r.ref_batch()
    return {"value": keys / dt, "unit": "keys/s", "cores": workers, "kind": "reference",
            "sample": f"{steps} steps x {lanes} lanes x {iters} batches of {r.ref_batch()} keys; the reference's "
                      f"src/gpu/common.h walk_thread compiled for the host, {workers} threads",
            "ms_per_step": dt / steps * 1e3}


def reference_cuda_kernel(b, lx, prefix: str) -> dict | None:
    """The reference's own CUDA kernel (src/gpu/kernel.cu + common.h, BATCH 64,
    block 128, SMs x 2048 threads as src/gpu/cuda.rs runs it) on this GPU, on
    the same prefix, with seeded starts whose first public keys come from
    lxmfv_first_public_keys."""
    from oracle import oracle as O
    if O.ref_cuda() is None:
        return None
    threads = O.ref_cuda().refcu_default_threads()
    setup = lx.seeded_setup(SEED + 77, threads)
    upc = b.first_public_keys(setup.scalars)
    r = O.ref_cuda_walk(upc, 64, 1, 3, setup.ed_pub, lx.name_hash(), lx.prefix_parse(prefix))
    return {"value": r["keys_per_s"], "unit": "keys/s", "threads": threads, "ms_per_launch": r["ms_per_launch"],
            "sample": "3 timed launches of 64 batches of 64 keys per thread (CUDA events), after 1 warm-up",
            "build": "reference src/gpu/kernel.cu + common.h, nvcc -gencode arch=compute_100a,code=sm_100a -O3"}


def batched_workload(lx, dev: int, single_value: float) -> dict:
    """256 concurrent searches in the pool's persistent kernel: prefix lengths
    uniform over 4-10 nibbles with random hex, aspects uniform over three, each
    with its own seeded identity; 1184 lanes each, so that the persistent
    kernel's work items (512 lanes) are exactly 4 per SM; G = 1024, 4 groups per
    step (the autotuned setting); aggregate device keys/s against the single
    search's `value`."""
    import lxmfv_serve as srv
    specs = srv.batched_specs(256, seed=4, lanes=1184, min_nibbles=4, max_nibbles=10)
    with srv.Pool(device=dev, capacity_lanes=256 * 1184, batch=1024) as pool:
        r = srv.run_batched(pool, specs, steps=6, groups=4, warmup=1)  # every hit rechecked
    r["vs_single_search"] = r["keys_per_s"] / single_value
    r["workload"] = "256 searches, 4-10 nibbles, 3 aspects, 1184 lanes each, one persistent launch per step"
    return r


def served_workload(dev: int, seconds: float) -> dict:
    """Served requests: Poisson arrivals at 50 per second for `seconds`, prefix
    length 5 + Geometric(0.9) - 1 truncated to 5-9 nibbles, random hex, aspects
    as in the batched workload, seeded identities; lanes by difficulty
    (64 x 16^(L-5), at most 32768); a pool of 262144 lanes (28 MB of walker
    state) as the memory budget; every search retired on its first hit."""
    import lxmfv_serve as srv
    reqs = srv.poisson_requests(rate=50.0, duration=seconds, seed=8, lanes=srv.lanes_by_difficulty)
    with srv.Pool(device=dev, capacity_lanes=262144, batch=256) as pool:
        out = srv.serve(pool, reqs, groups=1, time_limit=seconds + 240)
    out["workload"] = (f"Poisson 50 req/s for {seconds:.0f} s, 5-9 nibbles (geometric p=0.9), lanes by difficulty, "
                       "262144-lane pool")
    return out


def relaunch(n: int) -> int:
    """--gpus N > 1 without a launcher: start N ranks of this same command line
    under torch.distributed.run, one process per GPU, rendezvous on
    127.0.0.1; returns the launcher's exit code (non-zero if any rank
    failed).  Only rank 0 prints the JSON line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def gather_ranks(dist, world: int, rec: dict) -> list[dict]:
    """Every rank's record, in rank order, on every rank (one all-gather)."""
    if world == 1:
        return [rec]
    out: list = [None] * world
    dist.all_gather_object(out, rec)
    return out


def main() -> None:
    a = parse()
    if a.gpus < 1:
        sys.exit("bench.py: --gpus must be at least 1")
    if "WORLD_SIZE" not in os.environ and a.gpus > 1:
        sys.exit(relaunch(a.gpus))
    world, rank, local = dist_setup()
    if world != a.gpus:
        sys.exit(f"bench.py: --gpus {a.gpus} does not match the {world} rank(s) launched")
    if a.impl == "reference":
        if rank != 0:
            return
        prefix = _prefix()
        ref = reference_cpu(prefix, a.steps, a.warmup)
        line = {"metric": METRIC, "value": ref["value"], "unit": "keys/s", "n_gpus": a.gpus, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ref.get("ms_per_step"), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded ChaCha20 starts)",
                "impl": "reference",
                "config": {"workload": "plain search, host cores", "prefix": prefix, "batch": 64},
                "cpu_baseline": {"value": ref["value"], "unit": "keys/s", "cores": ref["cores"],
                                 "kind": ref["kind"], "sample": ref["sample"]},
                "e2e": {"value": ref["value"], "unit": "keys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    if a.engine != "gpu":
        host_engine_main(a, world, rank)
        return

    import torch
    import torch.distributed as dist

    import lxmfv as lx
    if torch.cuda.device_count() < world:
        sys.exit(f"bench.py: {world} ranks need {world} GPUs; {torch.cuda.device_count()} visible")
    dev = local
    torch.cuda.set_device(dev)  # before the process group, so each rank's NCCL communicator uses its own GPU
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    prefix = _prefix()
    head = measure(torch, dist, lx, a, dev, rank, world, prefix, a.walk, a.batch, a.total_keys, a.steps, a.warmup,
                   e2e=not a.no_e2e)
    ranks = gather_ranks(dist, world, head["rank_record"])
    line = {
        "metric": METRIC, "value": head["value"], "unit": "keys/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded ChaCha20 starts, numpy-seeded prefix)",
        "config": head["config"],
        "gpu_launches": a.steps,
        "e2e": head["e2e"],
        "roofline": head["roofline"],
        "clocks": head["clocks"],
        "hits": head["hits"],
        "ranks": ranks,
        "start_points_s": head["start_points_s"],
    }
    bad = head["hits"]["rechecked_bad"]
    # The side sections run once, on a single-GPU run (rank 0 of world 1).
    single = rank == 0 and world == 1
    if single and not a.no_b64 and a.batch != 64:
        # The same workload at B = 64 keys per inversion, the reference kernel's
        # batch: the grouped walk, then the x-only walk (the reference's
        # algorithm: xADD by Q and Montgomery batch inversion over 64 keys).
        # Each in its fastest launch shape (the autotuner's): the x-only walk runs
        # without the phase barrier, 3% faster than with it.
        for key, walk, shape in (("at_batch_64", "group", None), ("xadd_b64", "xadd", (512, False))):
            r = measure(torch, dist, lx, a, dev, rank, world, prefix, walk, 64, a.total_keys, a.steps, a.warmup,
                        e2e=False, shape=shape)
            line[key] = {"value": r["value"], "unit": "keys/s", "ms_per_step": r["ms_per_step"],
                         "gpu_launches": a.steps, "config": r["config"], "roofline": r["roofline"],
                         "clocks": r["clocks"], "hits": r["hits"]}
            bad += r["hits"]["rechecked_bad"]
    if single and not a.no_batched:
        line["batched"] = batched_workload(lx, dev, head["value"])
        bad += line["batched"]["rechecked_bad"]
    if single and a.served_seconds > 0:
        line["served"] = served_workload(dev, a.served_seconds)
        bad += line["served"]["rechecked_bad"]
    if single and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(prefix)
    if single and not a.no_cpu_search:
        line["cpu_search"] = cpu_search_rate()
    if single and not a.no_ref_cuda:
        with lx.Backend(device=dev, lanes=1024) as b:
            line["reference_cuda_kernel"] = reference_cuda_kernel(b, lx, prefix)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if bad:
        sys.exit(f"{bad} GPU hits failed their CPU recheck")


def host_engine_main(a, world: int, rank: int) -> None:
    """The multi-rank plumbing of the GPU run (rank seeds, max-over-ranks
    timing, the whole-job rate, one line from rank 0) around a host-side
    engine `module:function`, with gloo between the ranks.  The function is
    called as f(seed=, steps=, warmup=, prefix=, lanes=) and returns
    {"keys_per_step": K, "ms": device-or-wall milliseconds of the timed steps,
    "hits": [(lane, n), ...]}."""
    import datetime
    import importlib

    import torch.distributed as dist
    mod, _, fn = a.engine.partition(":")
    f = getattr(importlib.import_module(mod), fn)
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    seed = replicas.rank_seed(SEED, rank)
    prefix = _prefix()
    r = f(seed=seed, steps=a.steps, warmup=a.warmup, prefix=prefix, lanes=a.lanes or 4)
    ms = replicas.max_over_ranks(dist, r["ms"], "cpu")
    value = replicas.aggregate_rate(r["keys_per_step"] * a.steps, ms * 1e-3, world)
    ranks = gather_ranks(dist, world, {"rank": rank, "seed": seed, "ms": r["ms"], "hits": [list(h) for h in r["hits"]]})
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": value, "unit": "keys/s", "n_gpus": world, "steps": a.steps,
                          "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
                          "scaling": "weak", "engine": a.engine, "prefix": prefix, "ranks": ranks}), flush=True)


def measure(torch, dist, lx, a, dev, rank, world, prefix, walk, batch, total_keys, steps, warmup, e2e=True,
            shape: tuple[int, bool] | None = None) -> dict:
    """Times `steps` launches (after `warmup`) of the walk over `total_keys`
    keys in all, device-timed with CUDA events on the launching stream; every
    hit is rechecked from scratch on the CPU."""
    walk_id = lx.WALK_GROUP if walk == "group" else lx.WALK_XADD
    # A stream of our own (never the legacy default stream, whose handle is 0):
    # the library launches on it and the timing events are recorded on it.
    stream = torch.cuda.Stream(device=dev)
    # Launch shape: --block (0: the library's default), or the section's own (threads per block, phase barrier).
    block, flags = (shape[0], lx.FLAG_PHASE_SYNC if shape[1] else 0) if shape else (a.block, 0)
    with lx.Backend(device=dev, lanes=0, batch=batch, block=block, walk=walk_id, flags=flags) as b0:
        wave = b0.threads()
    lanes = a.lanes or wave * max(1, -(-131072 // wave))
    b = lx.Backend(device=dev, lanes=lanes, batch=batch, block=block, walk=walk_id, flags=flags,
                   stream=stream.cuda_stream)
    setup = lx.seeded_setup(replicas.rank_seed(SEED, rank), lanes)
    t0 = time.perf_counter()
    b.init_from_scalars(setup.scalars)
    ladder_s = time.perf_counter() - t0
    per_iter = lanes * batch
    iters = max(1, round(total_keys / (steps * per_iter)))
    keys_per_step = per_iter * iters
    args = lx.make_launch_args(iters, setup.ed_pub, lx.prefix_parse(prefix), max_hits=4096)

    for _ in range(warmup):
        b.launch_async(args)
    b.collect()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(dev) as clk:
        ev0.record(stream)
        for _ in range(steps):
            b.launch_async(args)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    ms_rank = ev0.elapsed_time(ev1)
    hits, n_hits = b.collect()
    ms = replicas.max_over_ranks(dist, ms_rank, f"cuda:{dev}")
    value = replicas.aggregate_rate(keys_per_step * steps, ms * 1e-3, world)

    # Every hit is rechecked from scratch on the CPU (OpenSSL), as the reference does.
    pfx = lx.prefix_parse(prefix)
    bad = [h for h in hits if not lx.prefix_matches(pfx, lx.address_of_identity(setup.identity(*h)))]

    # End to end through the C ABI: synchronous lxmfv_launch per step, launch
    # arguments from the host, hit count and hits read back every step.
    e2e_line = None
    if e2e:
        e2e_steps = max(1, steps // 2)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        d2h = 0
        for _ in range(e2e_steps):
            h, _, _, n = b.launch(args)
            d2h += 4 + 16 * len(h)
        dt = replicas.max_over_ranks(dist, time.perf_counter() - t0, f"cuda:{dev}")
        import ctypes
        e2e_line = {"value": replicas.aggregate_rate(keys_per_step * e2e_steps, dt, world), "unit": "keys/s",
                    "h2d_bytes_per_step": ctypes.sizeof(lx.LaunchArgs), "d2h_bytes_per_step": d2h // e2e_steps,
                    "steps": e2e_steps, "api": "lxmfv_launch (C ABI, synchronous, host buffers)"}

    imad_peak = b.peak_probe(0, 300.0)
    alu_peak = b.peak_probe(2, 300.0)
    b.close()
    kernel_s = ms * 1e-3 / steps
    mul, sqr = field_ops_per_key(walk, batch)
    prods = wide_products_per_key(walk, batch)
    keys_per_s_kernel = keys_per_step / kernel_s
    imad = 2 * prods * keys_per_s_kernel  # lo + hi IMAD per 32x32->64 product
    imad_line = {"achieved": imad / 1e12, "peak": imad_peak / 1e12, "unit": "T IMAD/s", "frac": imad / imad_peak,
                 "note": f"algorithmic {mul:.2f} M + {sqr:.2f} S = {prods:.0f} 32x32->64 products (lo + hi IMAD "
                         f"each) per key; peak = measured mad.lo.u32 rate of this GPU (probe)"}
    ncu = NCU_PER_KEY.get((walk, batch))
    if ncu:
        # The binding resource: the integer ALU pipe (SHA-256 rotates and LOP3s, carry handling).
        alu = ncu["alu"] * keys_per_s_kernel
        issue_peak = 2 * alu_peak  # 4 warp-instructions per SM per clock: twice the ALU pipe's lane rate
        roofline = {"bound": "alu", "achieved": alu / 1e12, "peak": alu_peak / 1e12, "unit": "T ALU lane-ops/s",
                    "frac": alu / alu_peak, "traffic": ncu["dram_bytes"] * keys_per_step,
                    "note": f"{ncu['alu']} ALU-pipe lane-ops per key (ncu, profiles/) x keys/s over the measured "
                            f"xor + funnel-shift rate of this GPU (probe); traffic = ncu DRAM bytes per key x keys "
                            f"per launch",
                    "issue": {"achieved": ncu["inst"] * keys_per_s_kernel / 1e12, "peak": issue_peak / 1e12,
                              "unit": "T inst/s", "frac": ncu["inst"] * keys_per_s_kernel / issue_peak},
                    "imad": imad_line}
        if "imad" in ncu:
            # The metric's own IMAD fraction: IMAD-class instructions per key
            # from ncu x keys/s over the measured mad.lo.u32 rate.
            imad_ncu = ncu["imad"] * keys_per_s_kernel
            roofline["imad_ncu"] = {"achieved": imad_ncu / 1e12, "peak": imad_peak / 1e12, "unit": "T IMAD/s",
                                    "frac": imad_ncu / imad_peak, "per_key": ncu["imad"],
                                    "note": "IMAD-class instructions per key from ncu (FMA-heavy pipe "
                                            "instructions x 32 / keys: IMAD, IMAD.HI, IMAD.WIDE, IMAD.X) x keys/s; "
                                            "peak = measured mad.lo.u32 rate of this GPU (probe)"}
    else:
        roofline = dict(imad_line, bound="imad", traffic=None, alu_peak=alu_peak / 1e12)
    config = {"workload": "plain GPU search (8-hex prefix, lxmf.delivery, seeded walkers, 2^36 keys per run)",
              "walk": walk, "prefix": prefix, "lanes_per_gpu": lanes, "batch": batch, "iters_per_step": iters,
              "block": block or 512, "phase_barrier": bool(flags) if block else True,
              "keys_per_step_per_gpu": keys_per_step, "parallelism": f"replicas x{world}",
              "l2": "working set (lane state + per-lane batch buffers) exceeds L2; no flush needed"}
    rank_record = {"rank": rank, "device": dev, "seed": replicas.rank_seed(SEED, rank), "ms": ms_rank,
                   "keys": keys_per_step * steps, "hits": int(n_hits), "rechecked_bad": len(bad)}
    return {"value": value, "ms_per_step": ms / steps, "e2e": e2e_line, "roofline": roofline,
            "clocks": clk.summary(), "hits": {"found": int(n_hits), "rechecked": len(hits), "rechecked_bad": len(bad)},
            "start_points_s": ladder_s, "config": config, "rank_record": rank_record}


def _prefix() -> str:
    """The workload's 8-hex-digit prefix: numpy's default_rng(SEED)."""
    import numpy as np
    rng = np.random.default_rng(SEED)
    return "".join("0123456789abcdef"[x] for x in rng.integers(0, 16, 8))


if __name__ == "__main__":
    main()
