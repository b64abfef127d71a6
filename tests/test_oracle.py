"""The oracle (CPU restatement) pinned against the reference's known answers,
its own tests (src/main.rs:501-563), the committed golden fixtures and,
where the reference tree was present to build it, the reference's own
common.h run on the CPU."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def kat():
    return json.load(open(os.path.join(GOLDEN, "kat.json")))


def test_address_matches_reticulum_for_a_known_identity(oracle):
    # main.rs:510-525: an identity made by RNS 1.5.7 and its rnid address.
    k = kat()
    assert oracle.address_of_identity(bytes.fromhex(k["identity"])).hex() == "b00b11fc764b58f813c3b3cc279f8b8a"


def test_u8b(oracle):
    assert oracle.u8b().hex() == kat()["u8b"]
    assert oracle.u8b().hex() == "6899c948ed6f71f11ea974adcaed787aa15cb6c84d883bd82d5cd6aad7a65f27"


def test_name_hash(oracle):
    import hashlib
    assert oracle.name_hash("lxmf.delivery") == hashlib.sha256(b"lxmf.delivery").digest()[:10]


def test_walked_public_keys_match_plain_x25519_across_batches(oracle):
    # main.rs:528-539: 3 batches of 256 from a start, each equal to x25519(k + 8n).
    k0, _, _ = oracle.seeded_identity(11)
    keys = oracle.walk_keys(k0, 3 * 256)
    for n in range(0, 3 * 256, 7):
        assert bytes(keys[n]) == oracle.x25519_base(oracle.step_scalar(k0, n)), n


def test_stepped_scalars_stay_clamped(oracle):
    # main.rs:542-553
    k0, _, _ = oracle.seeded_identity(5)
    for n in kat()["step_n"]:
        k = oracle.step_scalar(k0, n)
        assert k[0] & 7 == 0
        assert k[31] & 0xC0 == 0x40
    p = oracle.previous_scalar(k0)
    assert p[0] & 7 == 0 and p[31] & 0xC0 == 0x40
    assert oracle.step_scalar(p, 1) == k0


def test_prefixes_match_whole_and_half_bytes(oracle):
    # main.rs:556-562
    c = kat()["prefix_cases"]
    addr = bytes.fromhex(c["address"])
    for s in c["match"]:
        assert oracle.prefix_matches(oracle.prefix_parse(s), addr)
    for s in c["no_match"]:
        assert not oracle.prefix_matches(oracle.prefix_parse(s), addr)
    for s in c["invalid"]:
        assert oracle.prefix_parse(s) is None


def test_clamp_rejection_rule(oracle):
    # main.rs:164-169: bits 3..254 all clear, or bytes 9..31 all set, are rejected.
    ok, _ = oracle.clamp_start(bytes(32))
    assert not ok
    ok, _ = oracle.clamp_start(bytes(9) + b"\xff" * 23)
    assert not ok
    ok, k = oracle.clamp_start(b"\x07" + bytes(30) + b"\xff")
    assert ok and k[0] == 0 and k[31] == 0x7F


def test_seeding_convention_pinned(oracle):
    s = kat()["seed1"]
    k0, seed, off = oracle.seeded_identity(1)
    assert (k0.hex(), seed.hex(), off) == (s["scalar"], s["ed_seed"], s["offset"])
    more, _ = oracle.seeded_scalars(1, off, 4)
    assert [bytes(x).hex() for x in more] == s["scalars_1_4"]
    # RFC 8439 2.4.2 style check of the block function itself: key 0, counter 0.
    assert oracle.chacha20_stream(0, 0, 16).hex() == "76b8e0ada0f13d90405d6ae55386bd28"


def test_config1_window_prefix(oracle):
    """The first 2^16 keys of the seed-1 walk: hits and the first 4096
    destination hashes against the committed fixture."""
    c = json.load(open(os.path.join(GOLDEN, "config1.json")))
    k0, seed = bytes.fromhex(c["scalar"]), bytes.fromhex(c["ed_seed"])
    assert oracle.ed25519_public(seed).hex() == c["ed_pub"]
    hits, dump = oracle.search_window(k0, bytes.fromhex(c["ed_pub"]), bytes.fromhex(c["name_hash"]),
                                      oracle.prefix_parse(c["prefix"]), 1 << 19, dump=4096)
    assert [int(h) for h in hits] == [h for h in c["hits"] if h < (1 << 19)]
    gold = np.fromfile(os.path.join(GOLDEN, "config1_dest4096.bin"), np.uint8).reshape(4096, 16)
    assert (dump == gold).all()


@pytest.mark.slow
def test_config1_full_window(oracle):
    """All 2^24 keys of the seed-1 walk (about 25 s on one core)."""
    import hashlib
    c = json.load(open(os.path.join(GOLDEN, "config1.json")))
    hits, dump = oracle.search_window(bytes.fromhex(c["scalar"]), bytes.fromhex(c["ed_pub"]),
                                      bytes.fromhex(c["name_hash"]), oracle.prefix_parse(c["prefix"]), c["keys"],
                                      dump=4096)
    assert [int(h) for h in hits] == c["hits"]
    assert hashlib.sha256(dump.tobytes()).hexdigest() == c["dest4096_sha256"]


def test_field_small_golden(oracle):
    g = np.load(os.path.join(GOLDEN, "fe_small.npz"))
    assert (oracle.fe_op(0, g["a"], g["b"]) == g["mul"]).all()
    assert (oracle.fe_op(1, g["a"]) == g["sqr"]).all()
    assert (oracle.fe_op(2, g["a"]) == g["inv"]).all()
    assert (oracle.fe_batch_invert(g["a"], 64) == g["binv"]).all()


def test_field_against_python_integers(oracle):
    from tests.golden.inputs import EDGE, P, fe_inputs
    a, b = fe_inputs(64)
    val = lambda w: sum(int(x) << (32 * i) for i, x in enumerate(w))  # noqa: E731
    mul, sq, inv = oracle.fe_op(0, a, b), oracle.fe_op(1, a), oracle.fe_op(2, a)
    for i in range(64):
        x, y = val(a[i]) & ((1 << 255) - 1), val(b[i]) & ((1 << 255) - 1)
        assert val(mul[i]) == x * y % P
        assert val(sq[i]) == x * x % P
        assert val(inv[i]) == pow(x, P - 2, P)
    assert len(EDGE) > 10


def test_chain_small_golden(oracle):
    g = np.load(os.path.join(GOLDEN, "chain_small.npz"))
    assert (oracle.address_chain(g["pks"], oracle.name_hash("lxmf.delivery")) == g["out"]).all()


def test_chain_against_hashlib(oracle):
    import hashlib
    g = np.load(os.path.join(GOLDEN, "chain_small.npz"))
    nh = hashlib.sha256(b"lxmf.delivery").digest()[:10]
    for i in range(0, 256, 17):
        ih = hashlib.sha256(g["pks"][i].tobytes()).digest()[:16]
        assert hashlib.sha256(nh + ih).digest()[:16] == g["out"][i].tobytes()


def test_against_openssl(oracle):
    """X25519, Ed25519 and SHA-256 of the restatement against OpenSSL."""
    crypto = pytest.importorskip("cryptography.hazmat.primitives.asymmetric.x25519")
    from cryptography.hazmat.primitives import serialization
    from cryptography.hazmat.primitives.asymmetric import ed25519
    raw, rawf = serialization.Encoding.Raw, serialization.PublicFormat.Raw
    rng = np.random.default_rng(9)
    for _ in range(50):
        k, s = rng.bytes(32), rng.bytes(32)
        assert oracle.x25519_base(k) == crypto.X25519PrivateKey.from_private_bytes(k).public_key().public_bytes(raw, rawf)
        assert oracle.ed25519_public(s) == ed25519.Ed25519PrivateKey.from_private_bytes(s).public_key().public_bytes(raw, rawf)


def test_reference_build_agrees_with_restatement(oracle):
    """Where oracle/_ref exists: the reference's walk_thread on the CPU gives the
    same public keys and hits as the restatement."""
    import ctypes as C
    r = oracle.ref()
    if r is None:
        pytest.skip("oracle/_ref/libref.so not built here (needs the reference tree)")
    lanes = 3
    k0, es, off = oracle.seeded_identity(21)
    scal, _ = oracle.seeded_scalars(21, off, lanes - 1)
    starts = [k0] + [bytes(s) for s in scal]
    upc = np.zeros((lanes, 16), np.uint32)
    for t, k in enumerate(starts):
        upc[t, :8] = np.frombuffer(oracle.x25519_base(oracle.previous_scalar(k)), "<u4")
        upc[t, 8:] = np.frombuffer(oracle.x25519_base(k), "<u4")
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))  # noqa: E731
    state = np.zeros(lanes * 40, np.int32)
    ns = np.zeros(lanes, np.uint64)
    r.ref_init_walk(P(state, C.c_int32), P(upc, C.c_uint32), lanes)
    ed_pub = oracle.ed25519_public(es)
    ed = np.frombuffer(ed_pub, ">u4").astype(np.uint32)
    nh = oracle.name_hash()
    nhw = [int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)]
    pfx = oracle.prefix_parse("b0")
    w, m = oracle.prefix_words(pfx)
    want, mask = np.array(w, np.uint32), np.array(m, np.uint32)
    hc = np.zeros(1, np.uint32)
    hits = np.zeros(2 * 4096, np.uint64)
    dump = np.zeros(lanes * 64 * 8, np.uint32)
    q = np.frombuffer(oracle.u8b(), "<u4").astype(np.uint32)
    r.ref_walk(P(state, C.c_int32), P(ns, C.c_uint64), lanes, 3, P(ed, C.c_uint32), nhw[0], nhw[1], nhw[2],
               P(want, C.c_uint32), P(mask, C.c_uint32), P(hc, C.c_uint32), P(hits, C.c_uint64), 4096,
               P(dump, C.c_uint32), lanes, P(q, C.c_uint32))
    got = sorted((int(hits[2 * i]), int(hits[2 * i + 1])) for i in range(hc[0]))
    exp = []
    for t, k in enumerate(starts):
        h, _ = oracle.search_window(k, ed_pub, nh, pfx, 3 * 64)
        exp += [(t, int(n)) for n in h]
        assert (dump.reshape(lanes, 64, 8)[t].view(np.uint8).reshape(64, 32) == oracle.walk_keys(k, 64)).all()
    assert got == sorted(exp) and len(got) > 0
