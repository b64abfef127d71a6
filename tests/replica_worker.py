"""One rank of the replicated search on the CPU (gloo), for tests/test_replicas.py.

The rank's engine walks its seeded walkers with the library's CPU walk and
address chain (lxmfv_cpu_walk, lxmfv_cpu_addresses): the same keys and hashes
a GPU rank walks, at a size the CPU finishes in moments.  Prints one JSON line.

    python tests/replica_worker.py --rank R --world W --port P --case search|max|fail
"""
import argparse
import datetime
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "lxmf-vanity_b200"))

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

import lxmfv as lx  # noqa: E402
import lxmfv_replicas as rep  # noqa: E402


class CpuEngine:
    """Lanes of seeded walkers, `keys` keys per lane per launch, on this CPU."""

    def __init__(self, seed: int, lanes: int, keys: int, prefix: str, aspect: str, fail_at: int | None = None):
        self.setup = lx.seeded_setup(seed, lanes)
        self.prefix, self.aspect, self.keys = lx.prefix_parse(prefix), aspect, keys
        self.pos = 0
        self.launches = 0
        self.fail_at = fail_at

    def launch(self):
        self.launches += 1
        if self.fail_at is not None and self.launches >= self.fail_at:
            raise RuntimeError("injected engine failure")
        ed = np.frombuffer(self.setup.ed_pub, np.uint8)
        hits = []
        for lane, k in enumerate(self.setup.scalars):
            keys = lx.cpu_walk(lx.step_scalar(bytes(k), self.pos), self.keys)
            addrs = lx.cpu_addresses(np.concatenate([keys, np.tile(ed, (self.keys, 1))], 1), self.aspect)
            hits += [(lane, self.pos + i) for i in range(self.keys) if lx.prefix_matches(self.prefix, bytes(addrs[i]))]
        self.pos += self.keys
        return hits

    def identity(self, lane, n):
        return self.setup.identity(lane, n)

    def recheck(self, identity):
        return lx.prefix_matches(self.prefix, lx.address_of_identity(identity, self.aspect))


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--rank", type=int, required=True)
    p.add_argument("--world", type=int, required=True)
    p.add_argument("--port", type=int, required=True)
    p.add_argument("--case", choices=["search", "max", "fail"], required=True)
    p.add_argument("--seed", type=int, default=5)
    p.add_argument("--prefix", default="abc")
    p.add_argument("--aspect", default="lxmf.delivery")
    a = p.parse_args()
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{a.port}", rank=a.rank, world_size=a.world,
                            timeout=datetime.timedelta(seconds=60))
    out = {"rank": a.rank}
    try:
        if a.case == "max":
            out["max"] = rep.max_over_ranks(dist, 1.5 + a.rank)
            out["rate"] = rep.aggregate_rate(1000.0, out["max"], a.world)
        else:
            eng = CpuEngine(rep.rank_seed(a.seed, a.rank), lanes=4, keys=256, prefix=a.prefix, aspect=a.aspect,
                            fail_at=2 if (a.case == "fail" and a.rank == a.world - 1) else None)
            try:
                w = rep.replicated_search(dist, eng, max_rounds=64)
                out["winner"] = None if w is None else {"rank": w.rank, "lane": w.lane, "n": w.n,
                                                        "identity": w.identity.hex()}
            except RuntimeError as e:
                out["error"] = str(e)
            out["launches"] = eng.launches
    finally:
        dist.destroy_process_group()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
