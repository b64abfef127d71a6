"""Autotuner for the walk on this GPU.

Measures the plain search's keys/s for each launch configuration the library
builds and returns the fastest:

  - the walk: grouped (default) or x-only (the reference's);
  - keys per inversion: grouped G in {32, 64, 128, 256, 512, 1024}, x-only B in {16, 32, 64, 128};
  - threads per block: 128, 256 or 512, with or without the phase barrier;
  - the register cap: 128 per thread (every kernel) or 80 (LXMFV_FLAG_REGCAP_80:
    grouped walk, G = 256, 256-thread blocks with the barrier, three blocks per SM);
  - walk steps per launch (groups or batches per lane), for the fastest of the above,
    measured back to back so that launch gaps count.

The search pool's own sweep (keys per group and groups per step on a mix of
searches) is lxmfv_serve.autotune.

    python lxmf-vanity_b200/lxmfv_tune.py [--device 0] [--quick]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from dataclasses import asdict, dataclass

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lxmfv as lx  # noqa: E402

SEED = 3
PREFIX = "c1232cd9"


@dataclass(frozen=True)
class WalkConfig:
    walk: str   # "group" or "xadd"
    batch: int  # keys per inversion
    block: int  # threads per block
    sync: bool  # phase barrier
    regcap: int = 128
    ws: bool = False  # walker and hash warps (LXMFV_FLAG_WARP_SPEC)

    @property
    def flags(self) -> int:
        f = lx.FLAG_PHASE_SYNC if self.sync else 0
        f |= lx.FLAG_WARP_SPEC if self.ws else 0
        return f | (lx.FLAG_REGCAP_80 if self.regcap == 80 else 0)

    @property
    def walk_id(self) -> int:
        return lx.WALK_GROUP if self.walk == "group" else lx.WALK_XADD


def candidates(walks=("group", "xadd"), quick: bool = False) -> list[WalkConfig]:
    """Every configuration the library builds (a handful with `quick`)."""
    out = []
    shapes = [(128, False), (256, False), (256, True), (512, False), (512, True)]
    if "group" in walks:
        for g in ((512, 1024) if quick else (32, 64, 128, 256, 512, 1024)):
            for block, sync in (shapes if not quick else [(256, True), (512, True)]):
                out.append(WalkConfig("group", g, block, sync))
        out.append(WalkConfig("group", 256, 256, True, regcap=80))
        for g in (512, 1024):
            out.append(WalkConfig("group", g, 768, False, ws=True))
    if "xadd" in walks:
        for b in ((64, 128) if quick else (16, 32, 64, 128)):
            for block, sync in (shapes if not quick else [(512, True)]):
                out.append(WalkConfig("xadd", b, block, sync))
    return out


def measure(cfg: WalkConfig, device: int = 0, keys_per_launch: float = 2 ** 31, launches: int = 3,
            waves: int = 2) -> dict:
    """Kernel keys/s of one configuration: `waves` full waves of lanes, one
    warm-up launch, then the best of `launches` device-timed launches."""
    with lx.Backend(device=device, lanes=0, batch=cfg.batch, block=cfg.block, walk=cfg.walk_id,
                    flags=cfg.flags) as b0:
        wave = b0.threads()
    lanes = wave * waves
    with lx.Backend(device=device, lanes=lanes, batch=cfg.batch, block=cfg.block, walk=cfg.walk_id,
                    flags=cfg.flags) as b:
        setup = lx.seeded_setup(SEED, lanes)
        b.init_from_scalars(setup.scalars)
        iters = max(1, round(keys_per_launch / (lanes * cfg.batch)))
        args = lx.make_launch_args(iters, setup.ed_pub, lx.prefix_parse(PREFIX))
        b.launch(args)
        ms = []
        for _ in range(launches):
            b.launch(args)
            ms.append(b.last_kernel_ms())
    keys = lanes * cfg.batch * iters
    return {**asdict(cfg), "lanes": lanes, "iters": iters, "keys_per_s": keys / (min(ms) * 1e-3)}


def measure_steps(cfg: WalkConfig, device: int = 0, iters_list=(1, 4, 16, 64, 221), seconds: float = 1.5) -> list[dict]:
    """Back-to-back throughput of `cfg` for each walk-steps-per-launch count:
    asynchronous launches, timed by the host clock around the whole run, so
    launch gaps and tails count."""
    out = []
    with lx.Backend(device=device, lanes=0, batch=cfg.batch, block=cfg.block, walk=cfg.walk_id,
                    flags=cfg.flags) as b0:
        lanes = b0.threads() * 2
    with lx.Backend(device=device, lanes=lanes, batch=cfg.batch, block=cfg.block, walk=cfg.walk_id,
                    flags=cfg.flags) as b:
        setup = lx.seeded_setup(SEED, lanes)
        b.init_from_scalars(setup.scalars)
        for iters in iters_list:
            args = lx.make_launch_args(iters, setup.ed_pub, lx.prefix_parse(PREFIX))
            b.launch(args)  # warm-up; also the time of one launch
            one = max(b.last_kernel_ms(), 0.05)
            n = max(2, int(seconds * 1e3 / one))
            t0 = time.perf_counter()
            for _ in range(n):
                b.launch_async(args)
            b.collect()
            dt = time.perf_counter() - t0
            out.append({"iters": iters, "launches": n, "ms_per_launch": dt * 1e3 / n,
                        "keys_per_s": n * lanes * cfg.batch * iters / dt})
    return out


def tune(device: int = 0, walks=("group", "xadd"), quick: bool = False, keys_per_launch: float = 2 ** 31) -> dict:
    """Sweeps the configurations, then the steps per launch of the fastest."""
    results = []
    for cfg in candidates(walks, quick):
        try:
            results.append(measure(cfg, device, keys_per_launch=keys_per_launch))
        except lx.LxmfvError as e:
            results.append({**asdict(cfg), "error": str(e)})
    ok = [r for r in results if "keys_per_s" in r]
    best = max(ok, key=lambda r: r["keys_per_s"])
    cfg = WalkConfig(best["walk"], best["batch"], best["block"], best["sync"], best["regcap"], best["ws"])
    steps = measure_steps(cfg, device, iters_list=(1, 4, 16) if quick else (1, 4, 16, 64, 221))
    best_steps = max(steps, key=lambda r: r["keys_per_s"])
    return {"best": {**best, "iters": best_steps["iters"]}, "configs": results, "steps": steps}


def main() -> int:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--quick", action="store_true", help="a few configurations only")
    p.add_argument("--walk", choices=["group", "xadd", "both"], default="both")
    p.add_argument("--only", default=None,
                   help="measure one configuration, WALK:BATCH:BLOCK:SYNC[:ws] (e.g. group:1024:512:1 or "
                        "group:1024:768:0:ws), and print its line")
    p.add_argument("--keys-per-launch", type=float, default=2 ** 31)
    p.add_argument("--launches", type=int, default=3)
    a = p.parse_args()
    if a.only:
        f = a.only.split(":")
        cfg = WalkConfig(f[0], int(f[1]), int(f[2]), f[3] == "1", ws=len(f) > 4 and f[4] == "ws")
        print(json.dumps(measure(cfg, a.device, keys_per_launch=a.keys_per_launch, launches=a.launches)))
        return 0
    walks = ("group", "xadd") if a.walk == "both" else (a.walk,)
    r = tune(a.device, walks, a.quick)
    print(json.dumps(r))
    return 0


if __name__ == "__main__":
    sys.exit(main())
