"""Parity of the sm_100a kernels with the oracle, through the C ABI.

Bit-exact throughout: field primitives (mul, square, invert, batch
inversion) and the destination-hash chain against the golden fixtures;
public keys of the GPU ladder and of the walk against plain X25519; every
hit of the walk against the oracle's search; the seed-1 single-search window
(2^24 keys, prefix b00b1) split over lanes against its fixture."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _keys_of(dump: np.ndarray, lanes: int, keys: int) -> np.ndarray:
    return dump.reshape(lanes, keys, 8).view(np.uint8).reshape(lanes, keys, 32)


def _hashes_of(dump_addr: np.ndarray, lanes: int, keys: int) -> np.ndarray:
    return dump_addr.reshape(lanes, keys, 4).astype(">u4").view(np.uint8).reshape(lanes, keys, 16)


def test_describe(backend):
    d = backend.describe()
    assert "compute 10.0" in d and "SMs" in d
    assert backend.threads() == 4096 and backend.batch() == 64 and backend.walk() in (0, 1)


def test_field_small_golden(backend):
    g = np.load(os.path.join(GOLDEN, "fe_small.npz"))
    assert (backend.fe_op(0, g["a"], g["b"]) == g["mul"]).all()
    assert (backend.fe_op(1, g["a"]) == g["sqr"]).all()
    assert (backend.fe_op(2, g["a"]) == g["inv"]).all()
    assert (backend.fe_op(3, g["a"], group=64) == g["binv"]).all()


def test_field_digest(backend):
    from tests.golden.inputs import fe_inputs
    d = json.load(open(os.path.join(GOLDEN, "fe_digest.json")))
    a, b = fe_inputs(d["count"])
    dig = lambda x: hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest()  # noqa: E731
    assert dig(backend.fe_op(0, a, b)) == d["mul"]
    assert dig(backend.fe_op(1, a)) == d["sqr"]
    assert dig(backend.fe_op(2, a)) == d["inv"]
    assert dig(backend.fe_op(3, a, group=64)) == d["binv"]


def test_field_random_256bit_inputs(backend, oracle):
    """Full 256-bit inputs (bit 255 set included) against the oracle."""
    rng = np.random.default_rng(31)
    a = rng.integers(0, 2**32, size=(1 << 14, 8), dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 2**32, size=(1 << 14, 8), dtype=np.uint64).astype(np.uint32)
    a[:8] = 0xFFFFFFFF
    b[4:12] = 0xFFFFFFFF
    assert (backend.fe_op(0, a, b) == oracle.fe_op(0, a, b)).all()
    assert (backend.fe_op(1, a) == oracle.fe_op(1, a)).all()
    assert (backend.fe_op(2, a[:2048]) == oracle.fe_op(2, a[:2048])).all()
    for g in (1, 7, 64, 256):
        assert (backend.fe_op(3, a[:2048], group=g) == oracle.fe_batch_invert(a[:2048], g)).all(), g


def test_address_chain(backend, oracle):
    from tests.golden.inputs import chain_inputs
    g = np.load(os.path.join(GOLDEN, "chain_small.npz"))
    nh = oracle.name_hash("lxmf.delivery")
    assert (backend.address_chain(g["pks"], nh) == g["out"]).all()
    d = json.load(open(os.path.join(GOLDEN, "chain_digest.json")))
    out = backend.address_chain(chain_inputs(d["count"]), nh)
    assert hashlib.sha256(out.tobytes()).hexdigest() == d["sha256"]
    pks = chain_inputs(512)
    for aspect in ("nomadnetwork.node", "lxmf.propagation"):
        nh2 = oracle.name_hash(aspect)
        assert (backend.address_chain(pks, nh2) == oracle.address_chain(pks, nh2)).all()


def _walk(backend, lx, setup, prefix, iters, dump_lanes=0, dump_keys=0, max_hits=4096, aspect="lxmf.delivery"):
    args = lx.make_launch_args(iters, setup.ed_pub, lx.prefix_parse(prefix), aspect=aspect, max_hits=max_hits,
                               dump_threads=dump_lanes, dump_keys=dump_keys)
    return backend.launch(args, want_dump=dump_lanes > 0, want_dump_addr=dump_lanes > 0)


def test_ladder_start_points_and_first_batch(backend, lx, oracle):
    """GPU ladder starts: the first batch of every dumped lane equals
    x25519(k + 8i) (the shape of the reference's self-test, mod.rs:183-193)."""
    setup = lx.seeded_setup(101, backend.threads())
    backend.init_from_scalars(setup.scalars)
    hits, dump, dump_addr, n = _walk(backend, lx, setup, "b0", 1, dump_lanes=48)
    keys = _keys_of(dump, 48, 64)
    for t in range(48):
        k = bytes(setup.scalars[t])
        for i in range(0, 64, 3 if t > 2 else 1):
            assert bytes(keys[t, i]) == oracle.x25519_base(oracle.step_scalar(k, i)), (t, i)
    nh = oracle.name_hash()
    hashes = _hashes_of(dump_addr, 48, 64)
    for t in range(0, 48, 5):
        for i in range(64):
            assert bytes(hashes[t, i]) == oracle.lxmf_address(nh, bytes(keys[t, i]), setup.ed_pub)


def test_first_public_keys_match_x25519(backend, lx, oracle):
    """first_public_keys on the GPU: u(k-8), u(k) against plain X25519."""
    setup = lx.seeded_setup(111, 300)
    upc = backend.first_public_keys(setup.scalars)
    for t in range(0, 300, 7):
        k = bytes(setup.scalars[t])
        assert upc[t, :8].tobytes() == oracle.x25519_base(oracle.previous_scalar(k)), t
        assert upc[t, 8:].tobytes() == oracle.x25519_base(k), t
    with pytest.raises(lx.LxmfvError):
        backend.first_public_keys(np.zeros((2, 32), np.uint8))  # not clamped


def test_reference_cuda_kernel_agrees(backend, lx, oracle):
    """The reference's own walk kernel, built for sm_100a, and this one give
    the same hits and public keys for the same lanes."""
    if oracle.ref_cuda() is None:
        pytest.skip("oracle/_ref/libref_cuda.so not built (needs the reference tree)")
    lanes = backend.threads()
    setup = lx.seeded_setup(121, lanes)
    upc = backend.first_public_keys(setup.scalars)
    pfx = lx.prefix_parse("b00")
    r = oracle.ref_cuda_walk(upc, 4, 0, 1, setup.ed_pub, lx.name_hash(), pfx, dump_threads=8)
    backend.init(upc)
    hits, dump, _, n = _walk(backend, lx, setup, "b00", 4, dump_lanes=8)
    assert r["n_hits"] == n and sorted(r["hits"]) == sorted(hits) and n > 100
    assert (r["dump"] == dump).all()


def test_reference_init_interface(backend, lx, oracle):
    """Backend::init from u(k-8), u(k) words gives the same walk as the ladder."""
    lanes = backend.threads()
    setup = lx.seeded_setup(202, lanes)
    upc = np.zeros((lanes, 16), np.uint32)
    for t in range(lanes):
        k = bytes(setup.scalars[t])
        if t < 16:
            upc[t, :8] = np.frombuffer(oracle.x25519_base(oracle.previous_scalar(k)), "<u4")
            upc[t, 8:] = np.frombuffer(oracle.x25519_base(k), "<u4")
    backend.init(upc)
    _, dump_a, _, _ = _walk(backend, lx, setup, "b0", 2, dump_lanes=16, dump_keys=128)
    backend.init_from_scalars(setup.scalars)
    _, dump_b, _, _ = _walk(backend, lx, setup, "b0", 2, dump_lanes=16, dump_keys=128)
    assert (dump_a == dump_b).all()
    keys = _keys_of(dump_a, 16, 128)
    for t in range(16):
        walked = oracle.walk_keys(bytes(setup.scalars[t]), 128)
        assert (keys[t] == walked).all(), t


@pytest.mark.parametrize("batch,lanes", [(512, 512), (1024, 600)])
def test_warp_specialised_walk_matches_oracle(lx, oracle, batch, lanes):
    """Walker warps hand every key to hash warps through shared memory: the
    same keys, hashes and hits as the oracle, with a partial last block
    (600 lanes: 2 blocks of 256 and one of 88), across two launches."""
    with lx.Backend(device=0, lanes=lanes, batch=batch, flags=lx.FLAG_WARP_SPEC) as b:
        assert b.batch() == batch and b.threads() == lanes
        setup = lx.seeded_setup(909 + batch, lanes)
        b.init_from_scalars(setup.scalars)
        args = lx.make_launch_args(1, setup.ed_pub, lx.prefix_parse("b0"), max_hits=1 << 14, dump_threads=3,
                                   dump_keys=batch)
        hits1, dump1, addr1, n1 = b.launch(args, want_dump=True, want_dump_addr=True)
        hits2, dump2, _, n2 = b.launch(args, want_dump=True)
    nh = oracle.name_hash()
    keys1, keys2 = _keys_of(dump1, 3, batch), _keys_of(dump2, 3, batch)
    hashes = addr1.reshape(3, batch, 4).astype(">u4").view(np.uint8).reshape(3, batch, 16)
    for t in range(3):
        walked = oracle.walk_keys(bytes(setup.scalars[t]), 2 * batch)
        assert (keys1[t] == walked[:batch]).all() and (keys2[t] == walked[batch:]).all(), t
        for i in range(0, batch, 7):
            assert bytes(hashes[t, i]) == oracle.lxmf_address(nh, walked[i].tobytes(), setup.ed_pub)
    expected = set()
    for t in range(lanes):
        h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, nh, oracle.prefix_parse("b0"), 2 * batch)
        expected.update((t, int(x)) for x in h)
    assert set(hits1) | set(hits2) == expected and n1 + n2 == len(expected)


def test_warp_specialised_walk_refuses_other_shapes(lx):
    for kw in ({"batch": 256}, {"batch": 1024, "walk": lx.WALK_XADD}, {"batch": 1024, "block": 512}):
        with pytest.raises(lx.LxmfvError):
            lx.Backend(device=0, lanes=256, flags=lx.FLAG_WARP_SPEC, **kw)


def test_reference_init_interface_at_group_1024(lx, oracle):
    """The largest group (its table in constant memory): Backend::init from
    u(k-8), u(k) gives the oracle's keys, as the ladder start does."""
    lanes = 256
    with lx.Backend(device=0, lanes=lanes, batch=1024) as b:
        setup = lx.seeded_setup(212, lanes)
        upc = np.zeros((lanes, 16), np.uint32)
        for t in range(lanes):
            k = bytes(setup.scalars[t])
            upc[t, :8] = np.frombuffer(oracle.x25519_base(oracle.previous_scalar(k)), "<u4")
            upc[t, 8:] = np.frombuffer(oracle.x25519_base(k), "<u4")
        b.init(upc)
        _, dump_a, _, _ = _walk(b, lx, setup, "b0", 1, dump_lanes=4, dump_keys=1024)
        b.init_from_scalars(setup.scalars)
        _, dump_b, _, _ = _walk(b, lx, setup, "b0", 1, dump_lanes=4, dump_keys=1024)
    assert (dump_a == dump_b).all()
    keys = _keys_of(dump_a, 4, 1024)
    for t in range(4):
        assert (keys[t] == oracle.walk_keys(bytes(setup.scalars[t]), 1024)).all(), t


def test_hits_match_oracle_search(backend, lx, oracle):
    """Every hit of a 2-nibble search over 4096 lanes x 256 keys, exactly."""
    lanes = backend.threads()
    setup = lx.seeded_setup(303, lanes)
    backend.init_from_scalars(setup.scalars)
    hits, _, _, n = _walk(backend, lx, setup, "b0", 4, max_hits=1 << 16)
    assert n == len(hits)
    nh = oracle.name_hash()
    pfx = oracle.prefix_parse("b0")
    expected = set()
    for t in range(lanes):
        h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, nh, pfx, 256)
        expected.update((t, int(x)) for x in h)
    assert set(hits) == expected and len(hits) == len(expected)
    assert 3000 < len(expected) < 5200  # 2^20 keys / 256


def test_state_persists_across_launches(backend, lx, oracle):
    """Two launches continue one walk: indices 0..63 then 64..127."""
    setup = lx.seeded_setup(404, backend.threads())
    backend.init_from_scalars(setup.scalars)
    _, d1, _, _ = _walk(backend, lx, setup, "b0", 1, dump_lanes=4)
    _, d2, _, _ = _walk(backend, lx, setup, "b0", 1, dump_lanes=4)
    for t in range(4):
        walked = oracle.walk_keys(bytes(setup.scalars[t]), 128)
        assert (_keys_of(d1, 4, 64)[t] == walked[:64]).all()
        assert (_keys_of(d2, 4, 64)[t] == walked[64:]).all()


def test_config1_single_search_window(backend, lx):
    """Config 1: seed 1, lxmf.delivery, walk indices [0, 2^24), prefix b00b1,
    the walk split into 4096 lanes of 4096 keys.  All hits and the first 4096
    destination hashes against the fixture (oracle and reference agreed)."""
    c = json.load(open(os.path.join(GOLDEN, "config1.json")))
    lanes = backend.threads()
    per = c["keys"] // lanes
    setup = lx.segmented_setup(bytes.fromhex(c["scalar"]), bytes.fromhex(c["ed_seed"]), lanes, per)
    assert setup.ed_pub.hex() == c["ed_pub"]
    backend.init_from_scalars(setup.scalars)
    hits, _, dump_addr, n = _walk(backend, lx, setup, c["prefix"], per // 64, dump_lanes=1, dump_keys=4096)
    got = sorted(t * per + k for t, k in hits)
    assert got == c["hits"]
    gold = np.fromfile(os.path.join(GOLDEN, "config1_dest4096.bin"), np.uint8).reshape(4096, 16)
    assert (_hashes_of(dump_addr, 1, 4096)[0] == gold).all()
    for t, k in hits:
        assert lx.prefix_matches(lx.prefix_parse(c["prefix"]), lx.address_of_identity(setup.identity(t, k)))


def test_full_length_prefix_finds_exactly_one_key(backend, lx, oracle):
    """A 32-nibble prefix (the whole address) of one walked key: one hit."""
    setup = lx.seeded_setup(505, backend.threads())
    addr = oracle.lxmf_address(oracle.name_hash(), oracle.walk_keys(bytes(setup.scalars[7]), 200)[137].tobytes(),
                               setup.ed_pub)
    backend.init_from_scalars(setup.scalars)
    hits, _, _, n = _walk(backend, lx, setup, addr.hex(), 4)
    assert hits == [(7, 137)] and n == 1


def test_hit_queue_overflow_is_counted(backend, lx):
    setup = lx.seeded_setup(606, backend.threads())
    backend.init_from_scalars(setup.scalars)
    hits, _, _, n = _walk(backend, lx, setup, "b", 1, max_hits=5)
    assert len(hits) == 5 and n > 10000  # 2^18 keys / 16
    pfx = lx.prefix_parse("b")
    for t, k in hits:
        assert lx.prefix_matches(pfx, lx.address_of_identity(setup.identity(t, k)))


@pytest.mark.parametrize("aspect", ["nomadnetwork.node", "lxmf.propagation"])
def test_other_aspects(backend, lx, oracle, aspect):
    setup = lx.seeded_setup(707, backend.threads())
    backend.init_from_scalars(setup.scalars)
    hits, _, _, _ = _walk(backend, lx, setup, "c3", 1, aspect=aspect, max_hits=1 << 14)
    nh = oracle.name_hash(aspect)
    expected = set()
    for t in range(0, backend.threads()):
        h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, nh, oracle.prefix_parse("c3"), 64)
        expected.update((t, int(x)) for x in h)
    assert set(hits) == expected


@pytest.mark.parametrize("walk,batch,block", [(1, 16, 256), (1, 32, 128), (1, 128, 256),
                                              (0, 32, 256), (0, 128, 128), (0, 256, 256),
                                              (0, 512, 512), (0, 512, 256), (0, 1024, 512), (0, 1024, 128)])
def test_other_batch_sizes(lx, oracle, walk, batch, block):
    with lx.Backend(device=0, lanes=512, batch=batch, block=block, walk=walk) as b:
        assert b.walk() == walk and b.batch() == batch
        setup = lx.seeded_setup(808 + batch, 512)
        b.init_from_scalars(setup.scalars)
        args = lx.make_launch_args(2, setup.ed_pub, lx.prefix_parse("b0"), max_hits=1 << 14, dump_threads=3,
                                   dump_keys=2 * batch)
        hits, dump, _, n = b.launch(args, want_dump=True)
        keys = _keys_of(dump, 3, 2 * batch)
        for t in range(3):
            assert (keys[t] == oracle.walk_keys(bytes(setup.scalars[t]), 2 * batch)).all()
        expected = set()
        for t in range(512):
            h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, oracle.name_hash(),
                                        oracle.prefix_parse("b0"), 2 * batch)
            expected.update((t, int(x)) for x in h)
        assert set(hits) == expected


@pytest.mark.parametrize("block", [256, 512])
def test_phase_sync_with_a_partial_block(lx, oracle, block):
    """The block-barrier variant with lanes that do not fill the last block:
    the spare threads walk a copy of the last lane and must not emit or store."""
    lanes = 1000
    with lx.Backend(device=0, lanes=lanes, batch=64, block=block, flags=lx.FLAG_PHASE_SYNC) as b:
        setup = lx.seeded_setup(4242, lanes)
        b.init_from_scalars(setup.scalars)
        for launch in range(2):
            args = lx.make_launch_args(2, setup.ed_pub, lx.prefix_parse("a"), max_hits=1 << 14, dump_threads=lanes,
                                       dump_keys=128)
            hits, dump, _, n = b.launch(args, want_dump=True)
            assert n == len(hits)
            keys = _keys_of(dump, lanes, 128)
            for t in (0, 1, 511, 998, 999):
                walked = oracle.walk_keys(bytes(setup.scalars[t]), 256)
                assert (keys[t] == walked[128 * launch:128 * (launch + 1)]).all(), (t, launch)
            assert all(t < lanes for t, _ in hits)
            expected = set()
            for t in range(lanes):
                h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, oracle.name_hash(),
                                            oracle.prefix_parse("a"), 256)
                expected.update((t, int(x)) for x in h if 128 * launch <= x < 128 * (launch + 1))
            assert set(hits) == expected


def test_register_capped_kernel_matches_the_oracle(lx, oracle):
    """LXMFV_FLAG_REGCAP_80 (80 registers, three 256-thread blocks per SM):
    the same keys, hashes and hits as the oracle, over a partial last block
    and two launches."""
    lanes = 1000
    flags = lx.FLAG_PHASE_SYNC | lx.FLAG_REGCAP_80
    with lx.Backend(device=0, lanes=lanes, batch=256, block=256, flags=flags) as b:
        setup = lx.seeded_setup(5150, lanes)
        b.init_from_scalars(setup.scalars)
        for launch in range(2):
            args = lx.make_launch_args(1, setup.ed_pub, lx.prefix_parse("c"), max_hits=1 << 15, dump_threads=lanes,
                                       dump_keys=256)
            hits, dump, dump_addr, n = b.launch(args, want_dump=True, want_dump_addr=True)
            keys = _keys_of(dump, lanes, 256)
            for t in (0, 255, 256, 767, 999):
                walked = oracle.walk_keys(bytes(setup.scalars[t]), 512)
                assert (keys[t] == walked[256 * launch:256 * (launch + 1)]).all(), (t, launch)
            expected = set()
            for t in range(lanes):
                h, _ = oracle.search_window(bytes(setup.scalars[t]), setup.ed_pub, oracle.name_hash(),
                                            oracle.prefix_parse("c"), 512)
                expected.update((t, int(x)) for x in h if 256 * launch <= x < 256 * (launch + 1))
            assert set(hits) == expected and n == len(hits)


def test_autotuner_quick_sweep(lx):
    import lxmfv_tune as tune
    cfgs = [tune.WalkConfig("group", 256, 512, True), tune.WalkConfig("group", 256, 256, True, regcap=80),
            tune.WalkConfig("xadd", 128, 512, True)]
    rows = [tune.measure(c, 0, keys_per_launch=2 ** 28, launches=2) for c in cfgs]
    assert all(r["keys_per_s"] > 1e9 for r in rows), rows
    steps = tune.measure_steps(cfgs[0], 0, iters_list=(1, 8), seconds=0.5)
    assert [s["iters"] for s in steps] == [1, 8] and all(s["keys_per_s"] > 1e9 for s in steps)


def test_walks_agree_with_each_other(lx):
    """The grouped and x-only walks give identical hits and dumps for the same lanes."""
    out = []
    for walk in (lx.WALK_GROUP, lx.WALK_XADD):
        with lx.Backend(device=0, lanes=2048, batch=64, walk=walk) as b:
            setup = lx.seeded_setup(999, 2048)
            b.init_from_scalars(setup.scalars)
            args = lx.make_launch_args(3, setup.ed_pub, lx.prefix_parse("0"), max_hits=1 << 16, dump_threads=2,
                                       dump_keys=192)
            hits, dump, dump_addr, n = b.launch(args, want_dump=True, want_dump_addr=True)
            out.append((sorted(hits), dump, dump_addr, n))
    assert out[0][0] == out[1][0] and out[0][3] == out[1][3] > 20000
    assert (out[0][1] == out[1][1]).all() and (out[0][2] == out[1][2]).all()


def test_bad_step_point_rejected(backend, lx):
    setup = lx.seeded_setup(1, backend.threads())
    backend.init_from_scalars(setup.scalars)
    args = lx.make_launch_args(1, setup.ed_pub, lx.prefix_parse("b0"))
    args.q[0] ^= 1
    with pytest.raises(lx.LxmfvError) as e:
        backend.launch(args)
    assert e.value.code == lx.ERR_ARG


def test_self_test_shape(lx):
    """The reference's --gpu-self-test (mod.rs:178-207) on the default-sized
    device: the first batch (64 keys, the reference's BATCH) of 256 lanes against
    plain X25519, >= 100 hits for 'b0' with iters = 1, every hit rechecked from
    scratch on the CPU."""
    with lx.Backend(device=0, batch=64) as b:
        lanes = b.threads()
        assert lanes >= 256
        starts = np.stack([np.frombuffer(lx.random_start_scalar(), np.uint8) for _ in range(256)])
        scal = np.concatenate([starts, lx.seeded_setup(909, lanes - 256).scalars])
        b.init_from_scalars(scal)
        seed = lx.os_random(32)
        ed_pub = lx.ed25519_public(seed)
        args = lx.make_launch_args(1, ed_pub, lx.prefix_parse("b0"), dump_threads=256)
        hits, dump, _, n = b.launch(args, want_dump=True)
        keys = _keys_of(dump, 256, b.batch())
        for t in range(256):
            for i in range(b.batch()):
                assert bytes(keys[t, i]) == lx.x25519_base(lx.step_scalar(bytes(scal[t]), i))
        assert len(hits) >= 100
        pfx = lx.prefix_parse("b0")
        for t, k in hits:
            assert lx.prefix_matches(pfx, lx.address_of_identity(lx.step_scalar(bytes(scal[t]), k) + seed))
