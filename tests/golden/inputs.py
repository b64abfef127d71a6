"""Seeded inputs of the primitive microbench (field elements and 64-byte
public keys), regenerated identically by the fixture script and the tests.

Field elements: the ChaCha20 stream of seed 2 cut into 32-byte little-endian
values with bit 255 cleared, each redrawn while it is >= p (uniform mod p);
then the edge values 0, 1, 2, p-1, p-2, 2^255-20 and values >= p (p,
p+1, 2^255-1, and the same with bit 255 set, which the reference drops)
overwrite the first slots of `a` and, rotated, of `b`.
Public keys: the ChaCha20 stream of seed 3 cut into 64-byte blocks.
"""
from __future__ import annotations

import numpy as np

P = 2**255 - 19
EDGE = [0, 1, 2, P - 1, P - 2, 2**255 - 20, P, P + 1, P + 18, 2**255 - 1,
        2**256 - 1, 2**255, 2**255 + 1, 2**255 + P - 1]


def _stream(seed: int, nbytes: int) -> bytes:
    from oracle import oracle as O
    return O.chacha20_stream(seed, 0, nbytes)


def _words(x: int) -> list[int]:
    return [(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)]


def fe_inputs(count: int) -> tuple[np.ndarray, np.ndarray]:
    raw = np.frombuffer(_stream(2, 2 * count * 32 + 4096), np.uint8)
    vals = []
    pos = 0
    while len(vals) < 2 * count:
        x = int.from_bytes(raw[pos:pos + 32].tobytes(), "little") & ((1 << 255) - 1)
        pos += 32
        if x < P:
            vals.append(x)
    arr = np.array([_words(v) for v in vals], np.uint32)
    a, b = arr[:count].copy(), arr[count:].copy()
    for i, e in enumerate(EDGE[: count]):
        a[i] = _words(e)
        b[(i + 3) % count] = _words(EDGE[(i + 5) % len(EDGE)])
    return a, b


def chain_inputs(count: int) -> np.ndarray:
    return np.frombuffer(_stream(3, 64 * count), np.uint8).reshape(count, 64).copy()
