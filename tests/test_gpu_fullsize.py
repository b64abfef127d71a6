"""The primitive microbench at its full size: 2^26 field elements through
multiply, square, inversion and the 64-element batch inversion, and 2^26
public keys through the destination-hash chain, on the GPU through the C ABI.

At this size the oracle cannot recompute everything in test time, so the
checks are properties that hold at any size, computed by the library itself,
plus a strided sample against the oracle:
  - a * a^-1 = 1 for every element that is not 0 mod p (and a^-1 = 0 for those);
  - a^2 equals a * a, and the batch inversion equals the single inversions in
    every group without a zero element;
  - every 1024th element (and every salted edge value) of each op, every 1024th
    group of the batch inversion and every 1024th destination hash equal the
    oracle's.
Inputs are uniform 255-bit values with the edge values (0, 1, 2, p-1, p-2,
2^255-20, values in [p, 2^255)) salted into every chunk; the elements are
processed in four calls of 2^24."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = (1 << 255) - 19
TOTAL = 1 << 26
CHUNK = 1 << 24
EDGE = [0, 1, 2, P - 1, P - 2, (1 << 255) - 20, P, P + 1, (1 << 255) - 1]


def _words(x: int) -> np.ndarray:
    return np.array([(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)], np.uint32)


def _value(w) -> int:
    return sum(int(v) << (32 * i) for i, v in enumerate(w))


def _chunk(rng, n: int) -> np.ndarray:
    a = rng.integers(0, 1 << 32, size=(n, 8), dtype=np.uint64).astype(np.uint32)
    a[:, 7] &= 0x7FFFFFFF
    for i, e in enumerate(EDGE):
        a[i * 977 % n] = _words(e)
    return a


SALT = [i * 977 % CHUNK for i in range(len(EDGE))]


@pytest.fixture(scope="module")
def fe_backend(lx):
    with lx.Backend(device=0, lanes=256) as b:
        yield b


def test_field_ops_full_size(fe_backend, oracle):
    be = fe_backend
    rng = np.random.default_rng(2026)
    one = _words(1)
    is_zero = np.zeros(CHUNK, bool)
    for pos, e in zip(SALT, EDGE):
        is_zero[pos] = e % P == 0  # uniform draws are 0 mod p with probability 2^-255
    for c in range(TOTAL // CHUNK):
        a = _chunk(rng, CHUNK)
        b = _chunk(rng, CHUNK)
        mul = be.fe_op(0, a, b)
        sqr = be.fe_op(1, a)
        inv = be.fe_op(2, a)
        binv = be.fe_op(3, a, group=64)
        # Properties over every element.
        assert (be.fe_op(0, a, inv)[~is_zero] == one).all(), f"chunk {c}: a * a^-1 != 1"
        assert (inv[is_zero] == 0).all()
        assert (sqr == be.fe_op(0, a, a)).all(), f"chunk {c}: a^2 != a * a"
        groups_ok = ~is_zero.reshape(-1, 64).any(axis=1)
        assert (binv.reshape(-1, 64, 8)[groups_ok] == inv.reshape(-1, 64, 8)[groups_ok]).all()
        # A strided sample and every edge value against the oracle.
        idx = np.unique(np.concatenate([np.arange(0, CHUNK, 1024), SALT]))
        assert (mul[idx] == oracle.fe_op(0, a[idx], b[idx])).all()
        assert (sqr[idx] == oracle.fe_op(1, a[idx])).all()
        assert (inv[idx] == oracle.fe_op(2, a[idx])).all()
        gidx = np.arange(0, CHUNK // 64, 1024)
        ga = a.reshape(-1, 64, 8)[gidx].reshape(-1, 8)
        assert (binv.reshape(-1, 64, 8)[gidx].reshape(-1, 8) == oracle.fe_batch_invert(ga, 64)).all()
        del a, b, mul, sqr, inv, binv


def test_address_chain_full_size(fe_backend, oracle):
    rng = np.random.default_rng(2027)
    nh = oracle.name_hash("lxmf.delivery")
    for c in range(TOTAL // CHUNK):
        pks = rng.integers(0, 256, size=(CHUNK, 64), dtype=np.uint8)
        out = fe_backend.address_chain(pks, nh)
        idx = np.arange(c, CHUNK, 1024)
        assert (out[idx] == oracle.address_chain(pks[idx], nh)).all(), f"chunk {c}"
        # Distinct random inputs give distinct 128-bit hashes.
        assert len(np.unique(out[idx].view(np.uint64).reshape(-1, 2), axis=0)) == len(idx)
        del pks, out
