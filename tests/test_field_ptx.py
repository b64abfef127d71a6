"""The field library's inline PTX, executed by a CPU interpreter and checked
against Python integers mod p = 2^255 - 19 (no GPU needed).

Covers the representation contract the walk kernel relies on: every result
is a 256-bit value congruent to the exact result, fe_canon gives the unique
value in [0, p), and the generated file matches its generator."""
import os
import random
import subprocess
import sys

import pytest

sys.path.insert(0, os.path.dirname(__file__))
import ptx_emu  # noqa: E402

CSRC = os.path.join(os.path.dirname(__file__), "..", "lxmf-vanity_b200", "csrc")
P = 2**255 - 19
EDGE = [0, 1, 2, 19, 38, P - 2, P - 1, P, P + 1, 2**255 - 20, 2**255 - 1, 2**255, 2**255 + 18,
        2**256 - 39, 2**256 - 38, 2**256 - 2, 2**256 - 1, 2**128 - 1, 2**224]


@pytest.fixture(scope="module")
def blocks():
    src = open(os.path.join(CSRC, "fe25519_ptx.cuh")).read() + open(os.path.join(CSRC, "fe25519.cuh")).read()
    return ptx_emu.extract_asm_blocks(src)


def cases(n=300, seed=7):
    rng = random.Random(seed)
    vals = EDGE + [rng.getrandbits(256) for _ in range(n)] + [rng.randrange(P) for _ in range(n)]
    return vals


def call(blocks, name, *ins):
    lines, n_out = blocks[name]
    args = [0] * n_out
    for x in ins:
        args += ptx_emu.words(x)
    return ptx_emu.value(ptx_emu.run(lines, args)[:8])


def test_generated_file_is_current():
    out = subprocess.run([sys.executable, os.path.join(CSRC, "gen_fe_ptx.py")], capture_output=True, text=True, check=True)
    assert out.stdout == open(os.path.join(CSRC, "fe25519_ptx.cuh")).read()


def test_mul(blocks):
    vals = cases()
    rng = random.Random(3)
    for a in vals:
        b = rng.choice(vals)
        r = call(blocks, "fe_mul_ptx", a, b)
        assert 0 <= r < 2**256 and r % P == (a * b) % P, (hex(a), hex(b))
    for a in EDGE:
        for b in EDGE:
            r = call(blocks, "fe_mul_ptx", a, b)
            assert r % P == (a * b) % P


def test_sqr(blocks):
    for a in cases():
        r = call(blocks, "fe_sqr_ptx", a)
        assert 0 <= r < 2**256 and r % P == (a * a) % P, hex(a)


def test_add_sub(blocks):
    vals = cases(150)
    rng = random.Random(5)
    for a in vals:
        for b in (rng.choice(vals), 0, 2**256 - 1, 38, a):
            r = call(blocks, "fe_add", a, b)
            assert r % P == (a + b) % P
            r = call(blocks, "fe_sub", a, b)
            assert 0 <= r < 2**256 and r % P == (a - b) % P, (hex(a), hex(b))


def test_mul_small(blocks):
    lines, n_out = blocks["fe_mul_small"]
    for a in cases(150):
        for k in (121665, 1, 0, (1 << 26) - 1):
            out = ptx_emu.run(lines, [0] * n_out + ptx_emu.words(a) + [k])
            r = ptx_emu.value(out[:8])
            assert r % P == (a * k) % P


def test_canon(blocks):
    for a in cases():
        r = call(blocks, "fe_canon", a)
        assert r == a % P, hex(a)


@pytest.mark.parametrize("name,label,arity", [("fe_mul_ptx", "FOLDED", 2), ("fe_sqr_ptx", "FOLDED", 1),
                                              ("fe_add", "ADDED", 2), ("fe_sub", "SUBBED", 2)])
def test_rare_carry_branch(blocks, name, label, arity):
    """The last carry (borrow) chain of each block runs only when limb 0
    carries (borrows); the edge values take both sides, and both give the
    exact result."""
    lines, n_out = blocks[name]
    seen = {}
    for a in EDGE:
        for b in (EDGE if arity == 2 else [None]):
            ins = (a, b) if arity == 2 else (a,)
            args = [0] * n_out
            for x in ins:
                args += ptx_emu.words(x)
            r = ptx_emu.value(ptx_emu.run(lines, args, seen)[:8])
            want = {"fe_mul_ptx": lambda: a * b, "fe_sqr_ptx": lambda: a * a,
                    "fe_add": lambda: a + b, "fe_sub": lambda: a - b}[name]()
            assert 0 <= r < 2**256 and r % P == want % P, tuple(hex(x) for x in ins)
    assert seen.get((label, True), 0) > 0 and seen.get((label, False), 0) > 0, seen
