#!/usr/bin/env python3
"""Writes the golden fixtures under tests/golden/ (run in a checkout that has
the reference tree, so that oracle/_ref/libref.so can be built).

Every fixture is produced by the C restatement (oracle/liboracle.so) AND by
the reference's own src/gpu/common.h built for the host (oracle/_ref), and
written only when the two agree bit for bit:

  kat.json              known answers: the identity of src/main.rs:517 and its
                        address (main.rs:524), u(8B), the prefix cases of
                        main.rs:556-562, the stepped-scalar cases of
                        main.rs:542-553, the seed-1 identity of the seeding
                        convention.
  config1.json          the single CPU search: seed 1, aspect lxmf.delivery,
                        walk indices [0, 2^24), prefix b00b1 -> every matching
                        index, plus the SHA-256 of the 4096 first destination
                        hashes.
  config1_dest4096.bin  those 4096 destination hashes (16 bytes each).
  fe_small.npz          256 seeded field elements (uniform mod p, salted with
                        the edge values) through mul, square, invert and the
                        64-element batch inversion.
  fe_digest.json        SHA-256 digests of the same four outputs over 2^16
                        elements drawn the same way (inputs are regenerated
                        from the seed by tests).
  chain_small.npz       256 seeded 64-byte public keys -> destination hashes.
  chain_digest.json     digest of the chain over 2^16 seeded keys.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

from tests.golden.inputs import chain_inputs, fe_inputs  # noqa: E402

CONFIG1 = dict(seed=1, aspect="lxmf.delivery", keys=1 << 24, prefix="b00b1", dump=4096)


def ref_search_segmented(start: bytes, ed_pub: bytes, nh: bytes, prefix: str, keys: int, lanes: int = 256):
    """The reference's walk_thread over one walk split into `lanes` segments."""
    r = O.ref()
    B = r.ref_batch()
    per = keys // lanes
    assert per % B == 0
    upc = np.zeros((lanes, 16), np.uint32)
    for t in range(lanes):
        k = O.step_scalar(start, t * per)
        upc[t, :8] = np.frombuffer(O.x25519_base(O.previous_scalar(k)), "<u4")
        upc[t, 8:] = np.frombuffer(O.x25519_base(k), "<u4")
    state = np.zeros(lanes * 40, np.int32)
    ns = np.zeros(lanes, np.uint64)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    r.ref_init_walk(P(state, C.c_int32), P(upc, C.c_uint32), lanes)
    ed = np.frombuffer(ed_pub, ">u4").astype(np.uint32)
    nhw = [int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)]
    w, m = O.prefix_words(O.prefix_parse(prefix))
    want = np.array(w, np.uint32)
    mask = np.array(m, np.uint32)
    hc = np.zeros(1, np.uint32)
    hits = np.zeros(2 * 4096, np.uint64)
    q = np.frombuffer(O.u8b(), "<u4").astype(np.uint32)
    r.ref_bench_walk(os.cpu_count() or 1, P(state, C.c_int32), P(ns, C.c_uint64), lanes, per // B, P(ed, C.c_uint32),
                     nhw[0], nhw[1], nhw[2], P(want, C.c_uint32), P(mask, C.c_uint32), P(hc, C.c_uint32),
                     P(hits, C.c_uint64), 4096, P(q, C.c_uint32))
    return sorted(int(hits[2 * i]) * per + int(hits[2 * i + 1]) for i in range(int(hc[0])))


def ref_dest_hashes(start: bytes, ed_pub: bytes, nh: bytes, count: int) -> np.ndarray:
    """Destination hashes of walk indices [0, count) by the reference's lxmf_address."""
    r = O.ref()
    keys = O.walk_keys(start, count)  # checked against plain X25519 in tests
    u = np.ascontiguousarray(keys.view("<u4").reshape(count, 8))
    ed = np.tile(np.frombuffer(ed_pub, ">u4").astype(np.uint32), (count, 1))
    nhw = np.array([int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)],
                   np.uint32)
    out = np.zeros((count, 4), np.uint32)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))  # noqa: E731
    r.ref_lxmf_address(P(u), P(ed), P(nhw), P(out), count)
    return out.astype(">u4").view(np.uint8).reshape(count, 16)


def ref_fe(op: int, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    r = O.ref()
    a = np.ascontiguousarray(a, np.uint32)
    bb = np.ascontiguousarray(b if b is not None else a, np.uint32)
    out = np.zeros_like(a)
    P = lambda x: x.ctypes.data_as(C.POINTER(C.c_uint32))  # noqa: E731
    if op == 3:
        r.ref_fe_batch_invert(P(a), P(out), a.shape[0], 64)
    else:
        r.ref_fe_op(op, P(a), P(bb), P(out), a.shape[0])
    return out


def ref_chain(pks: np.ndarray, nh: bytes) -> np.ndarray:
    r = O.ref()
    n = pks.shape[0]
    u = np.ascontiguousarray(pks[:, :32]).view("<u4").reshape(n, 8).astype(np.uint32)
    ed = np.ascontiguousarray(pks[:, 32:]).view(">u4").reshape(n, 8).astype(np.uint32)
    nhw = np.array([int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)],
                   np.uint32)
    out = np.zeros((n, 4), np.uint32)
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint32))  # noqa: E731
    r.ref_lxmf_address(P(u), P(ed), P(nhw), P(out), n)
    return out.astype(">u4").view(np.uint8).reshape(n, 16)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    O.build()
    if not O.ref_available():
        sys.exit("oracle/_ref/libref.so is missing: the reference tree is needed to make the fixtures")

    # ---- known answers
    ident = bytes.fromhex("e83d9ecdcdd012692583bd66f997bd0fd074d1ff05c62e892c3b5abbf1dd867801cc1353acc"
                          "bf59a42a1b951c71c6454cda7e4b8252ae6a5cb7fa55bb0430442")
    kat_addr = O.address_of_identity(ident).hex()
    assert kat_addr == "b00b11fc764b58f813c3b3cc279f8b8a", kat_addr
    scalar0, ed_seed, off = O.seeded_identity(1)
    kat = {
        "identity": ident.hex(),
        "address": kat_addr,
        "u8b": O.u8b().hex(),
        "name_hash_lxmf_delivery": O.name_hash("lxmf.delivery").hex(),
        "prefix_cases": {"address": "b00b1e5f000000000000000000000000",
                         "match": ["B00B1E5", "b00b1e5f"], "no_match": ["b00b1e6"], "invalid": ["BOOB", "", "0" * 33]},
        "seed1": {"scalar": scalar0.hex(), "ed_seed": ed_seed.hex(), "offset": off,
                  "ed_pub": O.ed25519_public(ed_seed).hex(),
                  "scalars_1_4": [bytes(s).hex() for s in O.seeded_scalars(1, off, 4)[0]]},
        "step_n": [0, 1, 1000, 2**32 - 1, 2**64 // 16],
    }
    json.dump(kat, open(os.path.join(HERE, "kat.json"), "w"), indent=1)

    # ---- config 1
    t0 = time.time()
    ed_pub = O.ed25519_public(ed_seed)
    nh = O.name_hash(CONFIG1["aspect"])
    pfx = O.prefix_parse(CONFIG1["prefix"])
    hits, dump = O.search_window(scalar0, ed_pub, nh, pfx, CONFIG1["keys"], dump=CONFIG1["dump"])
    t1 = time.time()
    ref_hits = ref_search_segmented(scalar0, ed_pub, nh, CONFIG1["prefix"], CONFIG1["keys"])
    ref_dump = ref_dest_hashes(scalar0, ed_pub, nh, CONFIG1["dump"])
    t2 = time.time()
    assert [int(h) for h in hits] == ref_hits, (hits, ref_hits)
    assert (dump == ref_dump).all()
    for n in hits:
        addr = O.address_of_identity(O.step_scalar(scalar0, int(n)) + ed_seed)
        assert O.prefix_matches(pfx, addr)
    c1 = dict(CONFIG1)
    c1.update(scalar=scalar0.hex(), ed_seed=ed_seed.hex(), ed_pub=ed_pub.hex(), name_hash=nh.hex(),
              hits=[int(h) for h in hits], dest4096_sha256=digest(dump),
              seconds_oracle=round(t1 - t0, 1), seconds_reference=round(t2 - t1, 1))
    json.dump(c1, open(os.path.join(HERE, "config1.json"), "w"), indent=1)
    dump.tofile(os.path.join(HERE, "config1_dest4096.bin"))
    print("config1:", len(hits), "hits", f"oracle {t1 - t0:.1f}s, reference {t2 - t1:.1f}s")

    # ---- field primitives
    small_a, small_b = fe_inputs(256)
    outs = {}
    for op, name in ((0, "mul"), (1, "sqr"), (2, "inv"), (3, "binv")):
        mine = O.fe_batch_invert(small_a, 64) if op == 3 else O.fe_op(op, small_a, small_b)
        ref = ref_fe(op, small_a, small_b)
        assert (mine == ref).all(), name
        outs[name] = mine
    np.savez_compressed(os.path.join(HERE, "fe_small.npz"), a=small_a, b=small_b, **outs)
    big_a, big_b = fe_inputs(1 << 16)
    dig = {"count": 1 << 16}
    for op, name in ((0, "mul"), (1, "sqr"), (2, "inv"), (3, "binv")):
        mine = O.fe_batch_invert(big_a, 64) if op == 3 else O.fe_op(op, big_a, big_b)
        ref = ref_fe(op, big_a, big_b)
        assert (mine == ref).all(), name
        dig[name] = digest(mine)
    json.dump(dig, open(os.path.join(HERE, "fe_digest.json"), "w"), indent=1)

    # ---- address chain
    nh = O.name_hash("lxmf.delivery")
    pks = chain_inputs(256)
    out = O.address_chain(pks, nh)
    assert (out == ref_chain(pks, nh)).all()
    np.savez_compressed(os.path.join(HERE, "chain_small.npz"), pks=pks, out=out)
    pks = chain_inputs(1 << 16)
    out = O.address_chain(pks, nh)
    assert (out == ref_chain(pks, nh)).all()
    json.dump({"count": 1 << 16, "aspect": "lxmf.delivery", "sha256": digest(out)},
              open(os.path.join(HERE, "chain_digest.json"), "w"), indent=1)
    print("fixtures written")


if __name__ == "__main__":
    main()
