"""ctypes bindings to the CPU checkers: oracle/liboracle.so (the C restatement)
and oracle/_ref/libref.so (the reference's own src/gpu/common.h built for the
host).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline and reference legs, always as the checker or
as the timed CPU baseline, never as the thing measured on the GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)

_lib = None
_ref = None


def ref_dir() -> str:
    """Where the reference tree is: $LXMFV_REF_DIR, else a directory named
    `reference` beside the repository, else '' (not available)."""
    d = os.environ.get("LXMFV_REF_DIR", "")
    if not d:
        beside = os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
        d = beside if os.path.isfile(os.path.join(beside, "src", "gpu", "common.h")) else ""
    return d


def build() -> None:
    """Compile the checkers (the reference shim only where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={ref_dir()}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_x25519.argtypes = [_u8p, _u8p, _u8p]
        L.orc_x25519_base.argtypes = [_u8p, _u8p]
        L.orc_ladder_unclamped.argtypes = [_u8p, _u8p, _u8p]
        L.orc_ed25519_public.argtypes = [_u8p, _u8p]
        L.orc_sha256.argtypes = [_u8p, C.c_size_t, _u8p]
        L.orc_step_scalar.argtypes = [_u8p, _u8p, C.c_uint64]
        L.orc_previous_scalar.argtypes = [_u8p, _u8p]
        L.orc_clamp_start.argtypes = [_u8p]
        L.orc_clamp_start.restype = C.c_int
        L.orc_chacha20_stream.argtypes = [C.c_uint64, C.c_uint64, _u8p, C.c_size_t]
        L.orc_seeded_identity.argtypes = [C.c_uint64, _u8p, _u8p, _u64p]
        L.orc_seeded_identity.restype = C.c_uint64
        L.orc_seeded_scalars.argtypes = [C.c_uint64, C.c_uint64, _u8p, C.c_uint64]
        L.orc_seeded_scalars.restype = C.c_uint64
        L.orc_name_hash.argtypes = [_u8p, C.c_size_t, _u8p]
        L.orc_lxmf_address.argtypes = [_u8p, _u8p, _u8p, _u8p]
        L.orc_address_of_identity.argtypes = [_u8p, _u8p, _u8p]
        L.orc_prefix_parse.argtypes = [C.c_char_p, _u8p]
        L.orc_prefix_parse.restype = C.c_int
        L.orc_prefix_matches.argtypes = [_u8p, C.c_int, _u8p]
        L.orc_prefix_matches.restype = C.c_int
        L.orc_prefix_words.argtypes = [_u8p, C.c_int, _u32p, _u32p]
        L.orc_u8b.argtypes = [_u8p]
        L.orc_walk_keys.argtypes = [_u8p, C.c_uint64, _u8p]
        L.orc_search_window.argtypes = [_u8p, _u8p, _u8p, _u8p, C.c_int, C.c_uint64, _u64p, C.c_uint64, _u8p, C.c_uint64]
        L.orc_search_window.restype = C.c_uint64
        L.orc_fe_op.argtypes = [C.c_int, _u32p, _u32p, _u32p, C.c_uint64]
        L.orc_fe_batch_invert.argtypes = [_u32p, _u32p, C.c_uint64, C.c_int]
        L.orc_address_chain.argtypes = [_u8p, _u8p, _u8p, C.c_uint64]
        L.orc_bench_search.argtypes = [C.c_int, C.c_uint64, C.c_uint64, _u8p, C.c_int, _u64p, _u64p]
        L.orc_bench_search.restype = C.c_double
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's common.h built for the host (None when absent)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        L = C.CDLL(REF_SO)
        L.ref_batch.restype = C.c_int
        L.ref_init_walk.argtypes = [_i32p, _u32p, C.c_uint32]
        L.ref_walk.argtypes = [_i32p, _u64p, C.c_uint32, C.c_uint32, _u32p, C.c_uint32, C.c_uint32, C.c_uint32,
                               _u32p, _u32p, _u32p, _u64p, C.c_uint32, _u32p, C.c_uint32, _u32p]
        L.ref_lxmf_address.argtypes = [_u32p, _u32p, _u32p, _u32p, C.c_uint64]
        L.ref_fe_op.argtypes = [C.c_int, _u32p, _u32p, _u32p, C.c_uint64]
        L.ref_fe_batch_invert.argtypes = [_u32p, _u32p, C.c_uint64, C.c_int]
        L.ref_bench_walk.argtypes = [C.c_int, _i32p, _u64p, C.c_uint32, C.c_uint32, _u32p, C.c_uint32, C.c_uint32,
                                     C.c_uint32, _u32p, _u32p, _u32p, _u64p, C.c_uint32, _u32p]
        L.ref_bench_walk.restype = C.c_double
        _ref = L
    return _ref


REF_CUDA_SO = os.path.join(HERE, "_ref", "libref_cuda.so")
_ref_cuda = None


def ref_cuda():
    """The reference's own CUDA kernel built for sm_100a (None when absent)."""
    global _ref_cuda
    if _ref_cuda is None:
        if not os.path.exists(REF_CUDA_SO):
            return None
        L = C.CDLL(REF_CUDA_SO)
        L.refcu_walk.argtypes = [_u32p, C.c_uint32, C.c_uint32, C.c_int, C.c_int, _u32p, C.c_uint32, C.c_uint32,
                                 C.c_uint32, _u32p, _u32p, _u32p, C.POINTER(C.c_double), C.POINTER(C.c_float), _u32p,
                                 _u64p, C.c_uint32, _u32p]
        L.refcu_walk.restype = C.c_int
        L.refcu_default_threads.restype = C.c_int
        _ref_cuda = L
    return _ref_cuda


def ref_cuda_walk(u_prev_cur: np.ndarray, iters: int, warmup: int, steps: int, ed_pub: bytes, nh: bytes,
                  prefix: tuple[bytes, int], dump_threads: int = 0) -> dict:
    """Runs the reference's walk kernel on the GPU; keys/s, hits, dump."""
    L = ref_cuda()
    upc = np.ascontiguousarray(u_prev_cur, np.uint32).reshape(-1, 16)
    threads = upc.shape[0]
    ed = np.frombuffer(ed_pub, ">u4").astype(np.uint32)
    nhw = [int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)]
    w, m = prefix_words(prefix)
    want, mask = np.array(w, np.uint32), np.array(m, np.uint32)
    q = np.frombuffer(u8b(), "<u4").astype(np.uint32)
    rate, ms, n = C.c_double(0), C.c_float(0), C.c_uint32(0)
    hits = np.zeros(2 * 4096, np.uint64)
    dump = np.zeros(max(dump_threads, 1) * 64 * 8, np.uint32)
    rc = L.refcu_walk(_p(upc, _u32p), threads, iters, warmup, steps, _p(ed, _u32p), nhw[0], nhw[1], nhw[2],
                      _p(want, _u32p), _p(mask, _u32p), _p(q, _u32p), C.byref(rate), C.byref(ms), C.byref(n),
                      _p(hits, _u64p), dump_threads, _p(dump, _u32p))
    if rc != 0:
        raise RuntimeError(f"reference CUDA kernel: CUDA error {rc}")
    k = min(n.value, 4096)
    return {"keys_per_s": rate.value, "ms_per_launch": ms.value, "n_hits": n.value,
            "hits": [(int(hits[2 * i]), int(hits[2 * i + 1])) for i in range(k)],
            "dump": dump[: dump_threads * 64 * 8] if dump_threads else None, "threads": threads}


def _buf(b: bytes | bytearray | np.ndarray):
    if isinstance(b, np.ndarray):
        return b.ctypes.data_as(_u8p)
    return (C.c_uint8 * len(b)).from_buffer_copy(bytes(b))


def _p(arr: np.ndarray, t):
    return arr.ctypes.data_as(t)


# ---- single-value helpers (bytes in, bytes out)

def x25519_base(k: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_x25519_base(out, _buf(k))
    return bytes(out)


def x25519(k: bytes, u: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_x25519(out, _buf(k), _buf(u))
    return bytes(out)


def ladder_unclamped(k: bytes, u: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_ladder_unclamped(out, _buf(k), _buf(u))
    return bytes(out)


def ed25519_public(seed: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_ed25519_public(out, _buf(seed))
    return bytes(out)


def sha256(msg: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_sha256(_buf(msg) if msg else None, len(msg), out)
    return bytes(out)


def step_scalar(k: bytes, n: int) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_step_scalar(out, _buf(k), n)
    return bytes(out)


def previous_scalar(k: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_previous_scalar(out, _buf(k))
    return bytes(out)


def clamp_start(k: bytes) -> tuple[bool, bytes]:
    b = (C.c_uint8 * 32).from_buffer_copy(k)
    ok = lib().orc_clamp_start(b)
    return bool(ok), bytes(b)


def chacha20_stream(seed: int, offset: int, length: int) -> bytes:
    out = (C.c_uint8 * length)()
    lib().orc_chacha20_stream(seed, offset, out, length)
    return bytes(out)


def seeded_identity(seed: int) -> tuple[bytes, bytes, int]:
    """(scalar0, ed25519 seed, stream offset after them)."""
    k = (C.c_uint8 * 32)()
    s = (C.c_uint8 * 32)()
    off = C.c_uint64(0)
    lib().orc_seeded_identity(seed, k, s, C.byref(off))
    return bytes(k), bytes(s), off.value


def seeded_scalars(seed: int, offset: int, count: int) -> tuple[np.ndarray, int]:
    out = np.zeros((count, 32), np.uint8)
    end = lib().orc_seeded_scalars(seed, offset, _p(out, _u8p), count)
    return out, end


def name_hash(aspect: str | bytes = b"lxmf.delivery") -> bytes:
    a = aspect.encode() if isinstance(aspect, str) else aspect
    out = (C.c_uint8 * 10)()
    lib().orc_name_hash(_buf(a), len(a), out)
    return bytes(out)


def lxmf_address(nh: bytes, x_pub: bytes, ed_pub: bytes) -> bytes:
    out = (C.c_uint8 * 16)()
    lib().orc_lxmf_address(_buf(nh), _buf(x_pub), _buf(ed_pub), out)
    return bytes(out)


def address_of_identity(identity: bytes, aspect: str | bytes = b"lxmf.delivery") -> bytes:
    out = (C.c_uint8 * 16)()
    lib().orc_address_of_identity(_buf(identity), _buf(name_hash(aspect)), out)
    return bytes(out)


def prefix_parse(s: str) -> tuple[bytes, int] | None:
    b = (C.c_uint8 * 16)()
    n = lib().orc_prefix_parse(s.encode(), b)
    return None if n < 0 else (bytes(b), n)


def prefix_matches(prefix: tuple[bytes, int], address: bytes) -> bool:
    return bool(lib().orc_prefix_matches(_buf(prefix[0]), prefix[1], _buf(address)))


def prefix_words(prefix: tuple[bytes, int]) -> tuple[list[int], list[int]]:
    w = (C.c_uint32 * 4)()
    m = (C.c_uint32 * 4)()
    lib().orc_prefix_words(_buf(prefix[0]), prefix[1], w, m)
    return list(w), list(m)


def u8b() -> bytes:
    out = (C.c_uint8 * 32)()
    lib().orc_u8b(out)
    return bytes(out)


# ---- array helpers

def walk_keys(start: bytes, count: int) -> np.ndarray:
    """u(start + 8n) for n in [0, count), by the reference's KeyWalk algorithm."""
    out = np.zeros((count, 32), np.uint8)
    lib().orc_walk_keys(_buf(start), count, _p(out, _u8p))
    return out


def search_window(start: bytes, ed_pub: bytes, nh: bytes, prefix: tuple[bytes, int], count: int,
                  max_hits: int = 1 << 16, dump: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(matching walk indices, addresses of the first `dump` indices)."""
    hits = np.zeros(max(max_hits, 1), np.uint64)
    dump_addr = np.zeros((max(dump, 1), 16), np.uint8)
    n = lib().orc_search_window(_buf(start), _buf(ed_pub), _buf(nh), _buf(prefix[0]), prefix[1], count,
                                _p(hits, _u64p), max_hits, _p(dump_addr, _u8p), dump)
    if n > max_hits:
        raise ValueError(f"{n} hits exceed max_hits={max_hits}")
    return hits[:n].copy(), dump_addr[:dump].copy()


def fe_op(op: int, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint32)
    bb = np.ascontiguousarray(b if b is not None else a, np.uint32)
    out = np.zeros_like(a)
    lib().orc_fe_op(op, _p(a, _u32p), _p(bb, _u32p), _p(out, _u32p), a.shape[0])
    return out


def fe_batch_invert(a: np.ndarray, group: int = 64) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint32)
    out = np.zeros_like(a)
    lib().orc_fe_batch_invert(_p(a, _u32p), _p(out, _u32p), a.shape[0], group)
    return out


def address_chain(pks: np.ndarray, nh: bytes) -> np.ndarray:
    pks = np.ascontiguousarray(pks, np.uint8)
    out = np.zeros((pks.shape[0], 16), np.uint8)
    lib().orc_address_chain(_p(pks, _u8p), _buf(nh), _p(out, _u8p), pks.shape[0])
    return out


def bench_search(threads: int, keys_per_thread: int, seed: int, prefix: tuple[bytes, int]) -> tuple[float, int, int]:
    """The restated CPU search on `threads` threads: (keys/s, keys, hits)."""
    keys = C.c_uint64(0)
    hits = C.c_uint64(0)
    rate = lib().orc_bench_search(threads, keys_per_thread, seed, _buf(prefix[0]), prefix[1], C.byref(keys), C.byref(hits))
    return rate, keys.value, hits.value
