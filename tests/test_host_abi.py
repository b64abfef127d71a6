"""The C-ABI library on the CPU: it loads, exports every entry point that
include/lxmfv.h declares, and its host-side rules (the reference's
Prefix, step_scalar, previous_scalar, random_start_scalar, name_hash and
address_of_identity) agree with the oracle.  No kernel is launched."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "lxmfv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lxmfv_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported(lx):
    import ctypes
    names = header_functions()
    assert len(names) >= 28
    L = ctypes.CDLL(lx.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n
        assert n in lx.SIGNATURES, f"{n} has no ctypes signature"


def test_open_reports_errors_instead_of_aborting(lx):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lx.LxmfvError) as e:
        lx.Backend(device=0)
    assert e.value.code == lx.ERR_CUDA and "CUDA" in str(e.value)


def test_pool_open_reports_errors(lx):
    import torch

    import lxmfv_serve
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lx.LxmfvError) as e:
        lxmfv_serve.Pool(device=0)
    assert e.value.code == lx.ERR_CUDA
    with pytest.raises(lx.LxmfvError) as e:
        lxmfv_serve.Pool(device=0, batch=100)
    assert e.value.code == lx.ERR_ARG


def test_served_request_stream_is_seeded(lx):
    import lxmfv_serve
    a = lxmfv_serve.poisson_requests(50.0, 2.0, seed=4, lanes=32)
    b = lxmfv_serve.poisson_requests(50.0, 2.0, seed=4, lanes=32)
    assert [(r.arrival, r.spec.prefix, r.spec.aspect) for r in a] == [(r.arrival, r.spec.prefix, r.spec.aspect) for r in b]
    assert 60 < len(a) < 140
    assert all(5 <= r.spec.nibbles <= 9 for r in a)
    assert all(r.spec.aspect in lxmfv_serve.ASPECTS for r in a)


def test_bad_options_are_rejected(lx):
    with pytest.raises(lx.LxmfvError) as e:
        lx.Backend(batch=48)
    assert e.value.code == lx.ERR_ARG


def test_prefix_rules(lx, oracle):
    for s in ["b", "B0", "b00b1", "B00B1E5", "b00b1e5f", "0123456789abcdef0123456789ABCDEF", "f" * 31]:
        assert lx.prefix_parse(s) == oracle.prefix_parse(s)
        assert lx.prefix_words(lx.prefix_parse(s)) == oracle.prefix_words(oracle.prefix_parse(s))
    for s in ["", "BOOB", "g", "0" * 33, "b00b 1"]:
        with pytest.raises(ValueError):
            lx.prefix_parse(s)
    addr = bytes.fromhex("b00b1e5f000000000000000000000000")
    assert lx.prefix_matches(lx.prefix_parse("B00B1E5"), addr)
    assert lx.prefix_matches(lx.prefix_parse("b00b1e5f"), addr)
    assert not lx.prefix_matches(lx.prefix_parse("b00b1e6"), addr)
    rng = np.random.default_rng(4)
    for _ in range(300):
        a = rng.bytes(16)
        s = a.hex()[: rng.integers(1, 33)]
        if rng.random() < 0.5:
            s = s[:-1] + ("0" if s[-1] != "0" else "1")
        assert lx.prefix_matches(lx.prefix_parse(s), a) == oracle.prefix_matches(oracle.prefix_parse(s), a)


def test_scalar_rules(lx, oracle):
    rng = np.random.default_rng(5)
    for _ in range(50):
        ok, k = lx.clamp_start(rng.bytes(32))
        ok2, k2 = oracle.clamp_start(k)
        assert ok == ok2 and k == k2
        for n in [0, 1, 1000, 2**32 - 1, 2**64 // 16, 2**64 - 1]:
            assert lx.step_scalar(k, n) == oracle.step_scalar(k, n)
        assert lx.previous_scalar(k) == oracle.previous_scalar(k)
    assert not lx.clamp_start(bytes(32))[0]
    assert not lx.clamp_start(bytes(9) + b"\xff" * 23)[0]


def test_seeded_draws(lx, oracle):
    for seed in [0, 1, 2, 12345, 2**64 - 1]:
        ident, off = lx.seeded_identity(seed)
        k0, s, off2 = oracle.seeded_identity(seed)
        assert ident == k0 + s and off == off2
        a, e1 = lx.seeded_scalars(seed, off, 9)
        b, e2 = oracle.seeded_scalars(seed, off, 9)
        assert (a == b).all() and e1 == e2


def test_random_start_scalar(lx):
    ks = {lx.random_start_scalar() for _ in range(20)}
    assert len(ks) == 20
    for k in ks:
        assert k[0] & 7 == 0 and k[31] & 0xC0 == 0x40


def test_address_and_keys(lx, oracle):
    ident = bytes.fromhex("e83d9ecdcdd012692583bd66f997bd0fd074d1ff05c62e892c3b5abbf1dd867801cc1353acc"
                          "bf59a42a1b951c71c6454cda7e4b8252ae6a5cb7fa55bb0430442")
    assert lx.address_of_identity(ident).hex() == "b00b11fc764b58f813c3b3cc279f8b8a"
    rng = np.random.default_rng(6)
    for _ in range(30):
        ident = rng.bytes(64)
        for aspect in ["lxmf.delivery", "nomadnetwork.node", "lxmf.propagation"]:
            assert lx.address_of_identity(ident, aspect) == oracle.address_of_identity(ident, aspect)
        assert lx.x25519_base(ident[:32]) == oracle.x25519_base(ident[:32])
        assert lx.ed25519_public(ident[32:]) == oracle.ed25519_public(ident[32:])
    assert lx.name_hash("lxmf.delivery") == oracle.name_hash("lxmf.delivery")


def test_launch_args_packing(lx):
    a = lx.make_launch_args(3, bytes(range(32)), lx.prefix_parse("b00b1"), max_hits=7, dump_threads=2)
    assert a.iters == 3 and a.max_hits == 7 and a.dump_threads == 2
    assert list(a.ed)[0] == 0x00010203 and list(a.want) == [0xB00B1000, 0, 0, 0]
    assert list(a.mask) == [0xFFFFF000, 0, 0, 0]
    assert list(a.q) == lx.le_words(lx.U8B)


def test_register_cap_needs_its_configuration(lx):
    """LXMFV_FLAG_REGCAP_80 is checked before any device call (no GPU needed)."""
    for kw in ({"batch": 128, "block": 256}, {"batch": 256, "block": 512}, {"batch": 256, "block": 256, "walk": 1}):
        with pytest.raises(lx.LxmfvError, match="REGCAP_80"):
            lx.Backend(device=0, lanes=256, flags=lx.FLAG_PHASE_SYNC | lx.FLAG_REGCAP_80, **kw)
    with pytest.raises(lx.LxmfvError, match="REGCAP_80"):
        lx.Backend(device=0, lanes=256, batch=256, block=256, flags=lx.FLAG_REGCAP_80)
