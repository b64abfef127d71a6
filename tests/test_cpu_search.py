"""The CPU search (the reference's default mode, src/main.rs:230-323) through
the C ABI: lxmfv_cpu_walk, lxmfv_cpu_addresses and lxmfv_cpu_search.

Pinned to the golden single-search fixture (seed 1, prefix b00b1: the first
hit of the walk is index 391453; the 4096 first destination hashes) and
checked against the oracle's KeyWalk and address chain.  No GPU is used."""
import hashlib
import json
import os
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def config1():
    with open(os.path.join(GOLDEN, "config1.json")) as f:
        return json.load(f)


def use_walk(lx, monkeypatch, walk):
    """Select the CPU walk (scalar 5 x 51-bit, or the AVX-512 IFMA lanes);
    skips where this CPU has no IFMA."""
    monkeypatch.setenv("LXMFV_CPU_WALK", walk)
    try:
        lx.cpu_walk(bytes(lx.seeded_identity(1)[0][:32]), 1)
    except lx.LxmfvError as e:
        assert walk == "ifma" and e.code == lx.ERR_STATE
        pytest.skip("this CPU has no AVX-512 IFMA")


@pytest.mark.parametrize("walk", ["scalar", "ifma"])
def test_walk_matches_the_oracle(lx, monkeypatch, walk):
    """Both walks, across their group boundaries (256 keys scalar, 2048 on the
    IFMA lanes)."""
    use_walk(lx, monkeypatch, walk)
    for seed in (1, 2, 99):
        ident, _ = lx.seeded_identity(seed)
        for count in (0, 1, 255, 256, 257, 1000, 2047, 2048, 2049, 4500):
            got = lx.cpu_walk(ident[:32], count)
            assert got.shape == (count, 32)
            assert np.array_equal(got, O.walk_keys(ident[:32], count)), (seed, count)


def test_unknown_walk_is_refused(lx, monkeypatch):
    monkeypatch.setenv("LXMFV_CPU_WALK", "montgomery")
    with pytest.raises(lx.LxmfvError) as e:
        lx.cpu_walk(bytes(32), 1)
    assert e.value.code == lx.ERR_STATE
    with pytest.raises(lx.LxmfvError) as e:
        lx.CpuSearch(lx.prefix_parse("c3"), threads=1, seed=13).run()
    assert e.value.code == lx.ERR_STATE


def test_walk_keys_are_x25519_of_the_stepped_scalars(lx):
    ident, _ = lx.seeded_identity(5)
    keys = lx.cpu_walk(ident[:32], 40)
    for n in (0, 1, 7, 39):
        assert bytes(keys[n]) == O.x25519_base(O.step_scalar(ident[:32], n))


@pytest.mark.parametrize("impl", [0, 1, 2, 3, 4])
def test_addresses_match_the_oracle(lx, impl):
    rng = np.random.default_rng(impl)
    pks = rng.integers(0, 256, (3000, 64), dtype=np.uint8)
    for aspect in ("lxmf.delivery", "nomadnetwork.node"):
        try:
            got = lx.cpu_addresses(pks, aspect, impl=impl)
        except lx.LxmfvError as e:
            assert impl >= 2 and e.code == lx.ERR_STATE  # no SHA extensions / AVX-512F on this CPU
            pytest.skip("this CPU lacks the instructions of this implementation")
        assert np.array_equal(got, O.address_chain(pks, O.name_hash(aspect)))


@pytest.mark.parametrize("count", [1, 2, 15, 16, 17, 31, 33])
def test_addresses_ragged_counts(lx, count):
    """Counts that are not a multiple of the 16 keys the AVX-512 path hashes
    at once (its tail is padded), against the portable path and the oracle."""
    rng = np.random.default_rng(100 + count)
    pks = rng.integers(0, 256, (count, 64), dtype=np.uint8)
    want = O.address_chain(pks, O.name_hash("lxmf.propagation"))
    for impl in (0, 1, 3, 4):
        try:
            got = lx.cpu_addresses(pks, "lxmf.propagation", impl=impl)
        except lx.LxmfvError as e:
            assert e.code == lx.ERR_STATE
            continue
        assert np.array_equal(got, want), impl


def test_golden_destination_hashes(lx, config1):
    keys = lx.cpu_walk(bytes.fromhex(config1["scalar"]), config1["dump"])
    pks = np.concatenate([keys, np.tile(np.frombuffer(bytes.fromhex(config1["ed_pub"]), np.uint8), (len(keys), 1))], 1)
    dest = lx.cpu_addresses(pks, config1["aspect"])
    assert hashlib.sha256(dest.tobytes()).hexdigest() == config1["dest4096_sha256"]


def test_golden_first_hit(lx, config1):
    """One thread on seeded walker 0 = the fixture's single search: its first hit."""
    s = lx.CpuSearch(lx.prefix_parse(config1["prefix"]), threads=1, aspect=config1["aspect"], seed=config1["seed"])
    ident = s.run()
    n = config1["hits"][0]
    assert ident == O.step_scalar(bytes.fromhex(config1["scalar"]), n) + bytes.fromhex(config1["ed_seed"])
    assert s.tries == n + 1


@pytest.mark.parametrize("walker", [0, 3, 1000, 5000])
def test_seeded_walker_matches_the_oracle(lx, walker):
    """Thread 0 walks seeded walker `walker`: the first hit of the oracle's
    search over the same walk."""
    seed, prefix = 11, O.prefix_parse("c3")
    k0, ed_seed, off = O.seeded_identity(seed)
    start = k0 if walker == 0 else bytes(O.seeded_scalars(seed, off, walker)[0][walker - 1])
    hits, _ = O.search_window(start, O.ed25519_public(ed_seed), O.name_hash(), prefix, 4096)
    s = lx.CpuSearch(prefix, threads=1, seed=seed, first_walker=walker)
    got = s.run()
    assert got == O.step_scalar(start, int(hits[0])) + ed_seed
    assert s.tries == int(hits[0]) + 1


@pytest.mark.parametrize("walk", ["scalar", "ifma"])
@pytest.mark.parametrize("hasher", ["c", "ni", "x16"])
@pytest.mark.parametrize("prefix_text", ["c3", "e01"])
def test_every_hasher_finds_the_first_hit(lx, monkeypatch, walk, hasher, prefix_text):
    """Each walk with each of the search's hashers (portable C, SHA extensions
    in pairs, AVX-512 sixteen at a time) returns the oracle's first hit in walk
    order, with the same tries."""
    use_walk(lx, monkeypatch, walk)
    monkeypatch.setenv("LXMFV_CPU_HASH", hasher)
    seed, prefix = 13, O.prefix_parse(prefix_text)
    k0, ed_seed, _ = O.seeded_identity(seed)
    hits, _ = O.search_window(k0, O.ed25519_public(ed_seed), O.name_hash(), prefix, 8192)
    assert len(hits), "the window holds a hit"
    s = lx.CpuSearch(prefix, threads=1, seed=seed)
    try:
        got = s.run()
    except lx.LxmfvError as e:
        assert hasher != "c" and e.code == lx.ERR_STATE
        pytest.skip("this CPU lacks the instructions of this hasher")
    assert got == O.step_scalar(k0, int(hits[0])) + ed_seed
    assert s.tries == int(hits[0]) + 1


def test_unknown_hasher_is_refused(lx, monkeypatch):
    monkeypatch.setenv("LXMFV_CPU_HASH", "sha3")
    with pytest.raises(lx.LxmfvError) as e:
        lx.CpuSearch(lx.prefix_parse("c3"), threads=1, seed=13).run()
    assert e.value.code == lx.ERR_STATE


def test_many_threads_give_a_valid_identity(lx):
    for aspect in ("lxmf.delivery", "nomadnetwork.node"):
        s = lx.CpuSearch(lx.prefix_parse("b00"), threads=4, aspect=aspect)
        ident = s.run()
        assert O.prefix_matches(O.prefix_parse("b00"), O.address_of_identity(ident, aspect))
        assert s.tries > 0


def test_seeded_threads_walk_their_own_walkers(lx):
    seed = 21
    k0, ed_seed, off = O.seeded_identity(seed)
    starts = [k0] + [bytes(r) for r in O.seeded_scalars(seed, off, 3)[0]]
    s = lx.CpuSearch(lx.prefix_parse("d1"), threads=4, seed=seed)
    got = s.run()
    assert got[32:] == ed_seed
    assert O.prefix_matches(O.prefix_parse("d1"), O.address_of_identity(got))
    # The hit is a key of one of the four walks.
    x = O.x25519_base(got[:32])
    assert any(x in {bytes(k) for k in O.walk_keys(st, 4096)} for st in starts)


def test_stop_ends_the_search(lx):
    s = lx.CpuSearch(lx.prefix_parse("0123456789abcdef"), threads=2)
    threading.Timer(0.3, s.stop).start()
    t0 = time.time()
    assert s.run() is None
    assert time.time() - t0 < 10
    assert s.tries > 0


def test_bad_arguments(lx):
    import ctypes as C
    stop, tries, ident = C.c_int(0), C.c_uint64(0), (C.c_uint8 * 64)()
    pb = (C.c_uint8 * 16)()
    nh = (C.c_uint8 * 10)()
    f = lx.lib().lxmfv_cpu_search
    assert f(pb, 0, nh, 1, None, 0, C.byref(stop), C.byref(tries), ident) == lx.ERR_ARG   # no nibbles
    assert f(pb, 33, nh, 1, None, 0, C.byref(stop), C.byref(tries), ident) == lx.ERR_ARG  # too many
    assert f(pb, 2, nh, 0, None, 0, C.byref(stop), C.byref(tries), ident) == lx.ERR_ARG   # no threads
    assert f(pb, 2, nh, 1, None, 5, C.byref(stop), C.byref(tries), ident) == lx.ERR_ARG   # walker without seed
    assert f(pb, 2, nh, 1, None, 0, None, C.byref(tries), ident) == lx.ERR_ARG            # no stop flag
    assert lx.lib().lxmfv_cpu_walk(None, 4, None) == lx.ERR_ARG
    assert lx.lib().lxmfv_cpu_addresses(None, 0, nh, None, 5) == lx.ERR_ARG
