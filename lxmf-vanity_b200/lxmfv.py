"""Python bindings (ctypes) to liblxmfv.so, the B200 key-walk search.

`Backend` mirrors the reference's `trait Backend` (src/gpu/mod.rs:41-52) over
the C ABI of include/lxmfv.h: describe / threads / batch / init / launch,
with the same packing conventions as `LaunchArgs` (mod.rs:29-38).  The
host-rule helpers mirror src/main.rs (prefixes, scalars, addresses).

The library is the product: if it is missing, or the GPU is not a B200,
every call raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# LXMFV_LIB names another build of the library (e.g. a variant under test).
LIB_PATH = os.environ.get("LXMFV_LIB") or os.path.join(PKG, "liblxmfv.so")

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_NOMEM = -3
ERR_STATE = -4
ERR_RECHECK = -5
ERR_OVERFLOW = -6
WALK_GROUP = 0
WALK_XADD = 1
FLAG_PHASE_SYNC = 1
FLAG_REGCAP_80 = 2
FLAG_WARP_SPEC = 4

# u(8B), the step point of the walk (mod.rs:111): 32 LE bytes.
U8B = bytes.fromhex("6899c948ed6f71f11ea974adcaed787aa15cb6c84d883bd82d5cd6aad7a65f27")
ASPECT = "lxmf.delivery"
MAX_HITS = 4096


class LxmfvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"liblxmfv error {code}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("lanes", C.c_uint32), ("batch", C.c_uint32), ("block", C.c_uint32),
                ("walk", C.c_uint32), ("flags", C.c_uint32), ("stream", C.c_void_p)]


class LaunchArgs(C.Structure):
    _fields_ = [("iters", C.c_uint32), ("ed", C.c_uint32 * 8), ("name_hash", C.c_uint32 * 3),
                ("want", C.c_uint32 * 4), ("mask", C.c_uint32 * 4), ("q", C.c_uint32 * 8),
                ("max_hits", C.c_uint32), ("dump_threads", C.c_uint32), ("dump_keys", C.c_uint32)]


class Hit(C.Structure):
    _fields_ = [("thread", C.c_uint32), ("reserved", C.c_uint32), ("n", C.c_uint64)]


class PoolOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("capacity_lanes", C.c_uint32), ("memory_budget", C.c_uint64),
                ("batch", C.c_uint32), ("max_searches", C.c_uint32), ("max_hits", C.c_uint32),
                ("stream", C.c_void_p)]


class SearchDesc(C.Structure):
    _fields_ = [("ed", C.c_uint32 * 8), ("name_hash", C.c_uint32 * 3), ("want", C.c_uint32 * 4),
                ("mask", C.c_uint32 * 4), ("lanes", C.c_uint32)]


class PoolHit(C.Structure):
    _fields_ = [("search", C.c_uint32), ("lane", C.c_uint32), ("n", C.c_uint64)]


class PoolInfo(C.Structure):
    _fields_ = [("capacity_lanes", C.c_uint32), ("free_lanes", C.c_uint32), ("active_searches", C.c_uint32),
                ("active_lanes", C.c_uint32), ("batch", C.c_uint32), ("sms", C.c_uint32)]


_u8p = C.POINTER(C.c_uint8)
_u32p = C.POINTER(C.c_uint32)
_lib = None

# Every entry point of include/lxmfv.h, with its argument and return types.
SIGNATURES = {
    "lxmfv_open": ([C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int),
    "lxmfv_last_error": ([C.c_void_p], C.c_char_p),
    "lxmfv_describe": ([C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "lxmfv_threads": ([C.c_void_p], C.c_uint32),
    "lxmfv_batch": ([C.c_void_p], C.c_uint64),
    "lxmfv_walk": ([C.c_void_p], C.c_uint32),
    "lxmfv_init": ([C.c_void_p, _u32p, C.c_size_t], C.c_int),
    "lxmfv_init_from_scalars": ([C.c_void_p, _u8p, C.c_size_t], C.c_int),
    "lxmfv_first_public_keys": ([C.c_void_p, _u8p, C.c_size_t, _u32p], C.c_int),
    "lxmfv_launch": ([C.c_void_p, C.POINTER(LaunchArgs), C.POINTER(Hit), C.c_uint32, _u32p, _u32p, _u32p], C.c_int),
    "lxmfv_launch_async": ([C.c_void_p, C.POINTER(LaunchArgs)], C.c_int),
    "lxmfv_collect": ([C.c_void_p, C.POINTER(Hit), C.c_uint32, _u32p, _u32p, _u32p], C.c_int),
    "lxmfv_last_kernel_ms": ([C.c_void_p], C.c_float),
    "lxmfv_close": ([C.c_void_p], None),
    "lxmfv_prefix_parse": ([C.c_char_p, _u8p], C.c_int),
    "lxmfv_prefix_matches": ([_u8p, C.c_int, _u8p], C.c_int),
    "lxmfv_prefix_words": ([_u8p, C.c_int, _u32p, _u32p], None),
    "lxmfv_name_hash": ([C.c_char_p, _u8p], None),
    "lxmfv_step_scalar": ([_u8p, C.c_uint64, _u8p], None),
    "lxmfv_previous_scalar": ([_u8p, _u8p], None),
    "lxmfv_clamp_start": ([_u8p], C.c_int),
    "lxmfv_seeded_identity": ([C.c_uint64, _u8p], C.c_uint64),
    "lxmfv_seeded_scalars": ([C.c_uint64, C.c_uint64, _u8p, C.c_uint64], C.c_uint64),
    "lxmfv_os_random": ([_u8p, C.c_size_t], C.c_int),
    "lxmfv_ed25519_public": ([_u8p, _u8p], C.c_int),
    "lxmfv_x25519_base": ([_u8p, _u8p], C.c_int),
    "lxmfv_address_of_identity": ([_u8p, _u8p, _u8p], C.c_int),
    "lxmfv_fe_op": ([C.c_void_p, C.c_int, _u32p, _u32p, _u32p, C.c_uint64, C.c_uint32], C.c_int),
    "lxmfv_address_chain": ([C.c_void_p, _u8p, _u8p, _u8p, C.c_uint64], C.c_int),
    "lxmfv_peak_probe": ([C.c_void_p, C.c_int, C.c_float, C.POINTER(C.c_double)], C.c_int),
    "lxmfv_fe_batch_invert_static": ([C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p, C.c_char_p,
                                      C.c_size_t], C.c_int),
    "lxmfv_pool_open": ([C.POINTER(PoolOptions), C.POINTER(C.c_void_p)], C.c_int),
    "lxmfv_pool_last_error": ([C.c_void_p], C.c_char_p),
    "lxmfv_pool_info": ([C.c_void_p, C.POINTER(PoolInfo)], C.c_int),
    "lxmfv_pool_submit": ([C.c_void_p, C.POINTER(SearchDesc), _u8p, _u32p], C.c_int),
    "lxmfv_pool_submit_many": ([C.c_void_p, C.POINTER(SearchDesc), C.c_uint32, _u8p, _u32p, _u32p], C.c_int),
    "lxmfv_pool_retire": ([C.c_void_p, C.c_uint32], C.c_int),
    "lxmfv_pool_step": ([C.c_void_p, C.c_uint32], C.c_int),
    "lxmfv_pool_poll": ([C.c_void_p, C.POINTER(PoolHit), C.c_uint32, _u32p], C.c_int),
    "lxmfv_pool_keys_per_lane": ([C.c_void_p, C.c_uint32], C.c_uint64),
    "lxmfv_pool_last_step_ms": ([C.c_void_p], C.c_float),
    "lxmfv_pool_close": ([C.c_void_p], None),
    "lxmfv_cpu_addresses": ([_u8p, C.c_uint64, _u8p, _u8p, C.c_int], C.c_int),
    "lxmfv_cpu_walk": ([_u8p, C.c_uint64, _u8p], C.c_int),
    "lxmfv_cpu_search": ([_u8p, C.c_int, _u8p, C.c_int, C.POINTER(C.c_uint64), C.c_uint64, C.POINTER(C.c_int),
                          C.POINTER(C.c_uint64), _u8p], C.c_int),
}
STATIC_SCRATCH_ELEMS = 131072
STOPPED = 1
CPU_MAX_THREADS = 4096


def fe_batch_invert_static(d_a: int, d_out: int, count: int, group: int = 64, stream: int | None = None) -> None:
    """lxmfv_fe_batch_invert_static on device pointers (no device allocation;
    asynchronous on `stream`).  Raises LxmfvError with the library's message."""
    err = C.create_string_buffer(256)
    rc = lib().lxmfv_fe_batch_invert_static(d_a, d_out, count, group, stream, err, 256)
    if rc != OK:
        raise LxmfvError(rc, err.value.decode())


def lib():
    """Load liblxmfv.so (raises when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with python lxmf-vanity_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _b(data: bytes, n: int | None = None):
    if n is not None and len(data) != n:
        raise ValueError(f"expected {n} bytes, got {len(data)}")
    return (C.c_uint8 * len(data)).from_buffer_copy(data)


# ---- host rules (main.rs / mod.rs)

def prefix_parse(text: str) -> tuple[bytes, int]:
    """Prefix::parse (main.rs:206-216): (16 prefix bytes, nibbles)."""
    out = (C.c_uint8 * 16)()
    n = lib().lxmfv_prefix_parse(text.encode(), out)
    if n < 0:
        raise ValueError(f"'{text.lower()}' isn't 1 to 32 hex digits: use 0-9 and a-f only (zero, not the letter O).")
    return bytes(out), n


def prefix_matches(prefix: tuple[bytes, int], address: bytes) -> bool:
    return bool(lib().lxmfv_prefix_matches(_b(prefix[0], 16), prefix[1], _b(address, 16)))


def prefix_words(prefix: tuple[bytes, int]) -> tuple[list[int], list[int]]:
    w = (C.c_uint32 * 4)()
    m = (C.c_uint32 * 4)()
    lib().lxmfv_prefix_words(_b(prefix[0], 16), prefix[1], w, m)
    return list(w), list(m)


def name_hash(aspect: str = ASPECT) -> bytes:
    out = (C.c_uint8 * 10)()
    lib().lxmfv_name_hash(aspect.encode(), out)
    return bytes(out)


def name_hash_words(nh: bytes) -> list[int]:
    """The name hash as 3 big-endian words (mod.rs:113-117)."""
    return [int.from_bytes(nh[0:4], "big"), int.from_bytes(nh[4:8], "big"), (nh[8] << 24) | (nh[9] << 16)]


def step_scalar(k: bytes, n: int) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().lxmfv_step_scalar(_b(k, 32), n, out)
    return bytes(out)


def previous_scalar(k: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    lib().lxmfv_previous_scalar(_b(k, 32), out)
    return bytes(out)


def clamp_start(k: bytes) -> tuple[bool, bytes]:
    b = _b(k, 32)
    ok = lib().lxmfv_clamp_start(b)
    return bool(ok), bytes(b)


def seeded_identity(seed: int) -> tuple[bytes, int]:
    """(64-byte identity: scalar || Ed25519 seed, stream offset after it)."""
    out = (C.c_uint8 * 64)()
    off = lib().lxmfv_seeded_identity(seed, out)
    return bytes(out), off


def seeded_scalars(seed: int, offset: int, count: int) -> tuple[np.ndarray, int]:
    out = np.zeros((count, 32), np.uint8)
    end = lib().lxmfv_seeded_scalars(seed, offset, out.ctypes.data_as(_u8p), count)
    return out, end


def os_random(n: int) -> bytes:
    out = (C.c_uint8 * n)()
    if lib().lxmfv_os_random(out, n) != OK:
        raise OSError("no system randomness")
    return bytes(out)


def random_start_scalar() -> bytes:
    """random_start_scalar (main.rs:157-171)."""
    while True:
        ok, k = clamp_start(os_random(32))
        if ok:
            return k


def ed25519_public(seed: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    if lib().lxmfv_ed25519_public(_b(seed, 32), out) != OK:
        raise RuntimeError("Ed25519 key derivation failed")
    return bytes(out)


def x25519_base(k: bytes) -> bytes:
    out = (C.c_uint8 * 32)()
    if lib().lxmfv_x25519_base(_b(k, 32), out) != OK:
        raise RuntimeError("X25519 failed")
    return bytes(out)


def address_of_identity(identity: bytes, aspect: str = ASPECT) -> bytes:
    """address_of_identity (main.rs:191-197), from scratch on the CPU."""
    out = (C.c_uint8 * 16)()
    if lib().lxmfv_address_of_identity(_b(identity, 64), _b(name_hash(aspect), 10), out) != OK:
        raise RuntimeError("address recheck failed to run")
    return bytes(out)


def cpu_addresses(pks: np.ndarray, aspect: str = ASPECT, impl: int = 0) -> np.ndarray:
    """lxmf_address on the CPU for (n, 64) public keys; impl 0 the fastest available, 1 portable C,
    2 SHA extensions, 3 SHA extensions two keys at a time, 4 AVX-512F sixteen keys at a time."""
    pks = np.ascontiguousarray(pks, np.uint8)
    out = np.zeros((pks.shape[0], 16), np.uint8)
    rc = lib().lxmfv_cpu_addresses(pks.ctypes.data_as(_u8p), pks.shape[0], _b(name_hash(aspect), 10),
                                   out.ctypes.data_as(_u8p), impl)
    if rc != OK:
        raise LxmfvError(rc, "lxmfv_cpu_addresses failed")
    return out


def cpu_walk(start: bytes, count: int) -> np.ndarray:
    """KeyWalk on the CPU (main.rs:230-290): the keys u(k + 8n), n < count, as (count, 32) bytes."""
    out = np.zeros((count, 32), np.uint8)
    rc = lib().lxmfv_cpu_walk(_b(start, 32), count, out.ctypes.data_as(_u8p))
    if rc != OK:
        raise LxmfvError(rc, "lxmfv_cpu_walk failed")
    return out


class CpuSearch:
    """The CPU search (main.rs:292-323 on `threads` threads, as run_search).

    run() blocks until a hit or stop(); other threads may call stop() and
    read tries while it runs (the foreign call releases the GIL)."""

    def __init__(self, prefix: tuple[bytes, int], threads: int, aspect: str = ASPECT, seed: int | None = None,
                 first_walker: int = 0):
        self.prefix, self.threads, self.aspect = prefix, threads, aspect
        self.seed, self.first_walker = seed, first_walker
        self._stop = C.c_int(0)
        self._tries = C.c_uint64(0)

    def stop(self) -> None:
        self._stop.value = 1

    @property
    def tries(self) -> int:
        return self._tries.value

    def run(self) -> bytes | None:
        """The rechecked 64-byte identity, or None when stopped first."""
        ident = (C.c_uint8 * 64)()
        seed = C.byref(C.c_uint64(self.seed)) if self.seed is not None else None
        rc = lib().lxmfv_cpu_search(_b(self.prefix[0], 16), self.prefix[1], _b(name_hash(self.aspect), 10),
                                    self.threads, seed, self.first_walker, C.byref(self._stop),
                                    C.byref(self._tries), ident)
        if rc == STOPPED:
            return None
        if rc != OK:
            raise LxmfvError(rc, "lxmfv_cpu_search failed")
        return bytes(ident)


def le_words(b: bytes) -> list[int]:
    return [int.from_bytes(b[4 * i: 4 * i + 4], "little") for i in range(len(b) // 4)]


def be_words(b: bytes) -> list[int]:
    return [int.from_bytes(b[4 * i: 4 * i + 4], "big") for i in range(len(b) // 4)]


def make_launch_args(iters: int, ed_pub: bytes, prefix: tuple[bytes, int], aspect: str = ASPECT,
                     max_hits: int = MAX_HITS, dump_threads: int = 0, dump_keys: int = 0) -> LaunchArgs:
    """LaunchArgs as GpuSearch::launch packs them (mod.rs:124-136)."""
    a = LaunchArgs()
    a.iters = iters
    a.ed[:] = be_words(ed_pub)
    a.name_hash[:] = name_hash_words(name_hash(aspect))
    w, m = prefix_words(prefix)
    a.want[:] = w
    a.mask[:] = m
    a.q[:] = le_words(U8B)
    a.max_hits = max_hits
    a.dump_threads = dump_threads
    a.dump_keys = dump_keys
    return a


# ---- the Backend (mod.rs:41-52) over the C ABI

class Backend:
    """One open device: walker state for `threads()` lanes."""

    def __init__(self, device: int = 0, lanes: int = 0, batch: int = 0, block: int = 0, stream: int | None = None,
                 walk: int = 0, flags: int = 0):
        L = lib()
        o = Options(device, lanes, batch, block, walk, flags, stream)
        h = C.c_void_p()
        rc = L.lxmfv_open(C.byref(o), C.byref(h))
        self._h = h
        if rc != OK:
            msg = L.lxmfv_last_error(h).decode() if h.value else "open failed"
            L.lxmfv_close(h)
            self._h = None
            raise LxmfvError(rc, msg)

    def _check(self, rc: int) -> None:
        if rc != OK:
            raise LxmfvError(rc, lib().lxmfv_last_error(self._h).decode())

    def close(self) -> None:
        if self._h is not None:
            lib().lxmfv_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def describe(self) -> str:
        buf = C.create_string_buffer(256)
        lib().lxmfv_describe(self._h, buf, 256)
        return buf.value.decode()

    def threads(self) -> int:
        return lib().lxmfv_threads(self._h)

    def batch(self) -> int:
        return lib().lxmfv_batch(self._h)

    def walk(self) -> int:
        return lib().lxmfv_walk(self._h)

    def init(self, u_prev_cur: np.ndarray) -> None:
        """Backend::init: 16 LE words per lane, u(k-8) then u(k)."""
        a = np.ascontiguousarray(u_prev_cur, np.uint32).reshape(-1)
        self._check(lib().lxmfv_init(self._h, a.ctypes.data_as(_u32p), a.size))

    def init_from_scalars(self, scalars: np.ndarray | bytes) -> None:
        """Start points by the GPU ladder from 32-byte clamped scalars."""
        a = np.frombuffer(scalars, np.uint8) if isinstance(scalars, (bytes, bytearray)) else \
            np.ascontiguousarray(scalars, np.uint8).reshape(-1)
        self._check(lib().lxmfv_init_from_scalars(self._h, a.ctypes.data_as(_u8p), a.size))

    def first_public_keys(self, scalars: np.ndarray) -> np.ndarray:
        """u(k-8), u(k) per scalar on the GPU: (count, 16) LE words for init()."""
        s = np.ascontiguousarray(scalars, np.uint8).reshape(-1, 32)
        out = np.zeros((s.shape[0], 16), np.uint32)
        self._check(lib().lxmfv_first_public_keys(self._h, s.ctypes.data_as(_u8p), s.shape[0],
                                                  out.ctypes.data_as(_u32p)))
        return out

    def launch(self, args: LaunchArgs, hits_cap: int | None = None, want_dump: bool = False,
               want_dump_addr: bool = False) -> tuple[list[tuple[int, int]], np.ndarray | None, np.ndarray | None, int]:
        """Backend::launch: ((thread, n) hits, dump words, dump hashes, total hit count)."""
        cap = args.max_hits if hits_cap is None else hits_cap
        hits = (Hit * max(cap, 1))()
        n = C.c_uint32(0)
        dk = args.dump_keys or self.batch()
        dl = min(args.dump_threads, self.threads())
        dump = np.zeros(dl * dk * 8, np.uint32) if (want_dump and dl) else None
        dump_addr = np.zeros(dl * dk * 4, np.uint32) if (want_dump_addr and dl) else None
        self._check(lib().lxmfv_launch(self._h, C.byref(args), hits, cap, C.byref(n),
                                       dump.ctypes.data_as(_u32p) if dump is not None else None,
                                       dump_addr.ctypes.data_as(_u32p) if dump_addr is not None else None))
        got = min(n.value, cap, args.max_hits)
        return [(hits[i].thread, hits[i].n) for i in range(got)], dump, dump_addr, n.value

    def launch_async(self, args: LaunchArgs) -> None:
        self._check(lib().lxmfv_launch_async(self._h, C.byref(args)))

    def collect(self, hits_cap: int = MAX_HITS) -> tuple[list[tuple[int, int]], int]:
        hits = (Hit * max(hits_cap, 1))()
        n = C.c_uint32(0)
        self._check(lib().lxmfv_collect(self._h, hits, hits_cap, C.byref(n), None, None))
        got = min(n.value, hits_cap)
        return [(hits[i].thread, hits[i].n) for i in range(got)], n.value

    def last_kernel_ms(self) -> float:
        return lib().lxmfv_last_kernel_ms(self._h)

    # primitives
    def fe_op(self, op: int, a: np.ndarray, b: np.ndarray | None = None, group: int = 64) -> np.ndarray:
        a = np.ascontiguousarray(a, np.uint32)
        bb = np.ascontiguousarray(b, np.uint32) if b is not None else None
        out = np.zeros_like(a)
        self._check(lib().lxmfv_fe_op(self._h, op, a.ctypes.data_as(_u32p),
                                      bb.ctypes.data_as(_u32p) if bb is not None else None,
                                      out.ctypes.data_as(_u32p), a.shape[0], group))
        return out

    def address_chain(self, pks: np.ndarray, nh: bytes) -> np.ndarray:
        pks = np.ascontiguousarray(pks, np.uint8)
        out = np.zeros((pks.shape[0], 16), np.uint8)
        self._check(lib().lxmfv_address_chain(self._h, pks.ctypes.data_as(_u8p), _b(nh, 10),
                                              out.ctypes.data_as(_u8p), pks.shape[0]))
        return out

    def peak_probe(self, kind: int, ms: float = 200.0) -> float:
        r = C.c_double(0)
        self._check(lib().lxmfv_peak_probe(self._h, kind, ms, C.byref(r)))
        return r.value


@dataclass
class Identity:
    scalar: bytes
    seed: bytes

    @property
    def bytes(self) -> bytes:
        return self.scalar + self.seed


@dataclass
class WalkSetup:
    """Lane starts for one search: scalars[t] is lane t's first key."""
    ed_seed: bytes
    ed_pub: bytes
    scalars: np.ndarray = field(repr=False)

    def identity(self, lane: int, n: int) -> bytes:
        """GpuSearch::identity (mod.rs:139-144)."""
        return step_scalar(bytes(self.scalars[lane]), n) + self.ed_seed


def seeded_setup(seed: int, lanes: int) -> WalkSetup:
    """Lane 0 starts at the seeded identity's scalar; lane t at the t-th further draw."""
    ident, off = seeded_identity(seed)
    scal = np.zeros((lanes, 32), np.uint8)
    scal[0] = np.frombuffer(ident[:32], np.uint8)
    if lanes > 1:
        more, _ = seeded_scalars(seed, off, lanes - 1)
        scal[1:] = more
    return WalkSetup(ident[32:], ed25519_public(ident[32:]), scal)


def segmented_setup(start: bytes, ed_seed: bytes, lanes: int, keys_per_lane: int) -> WalkSetup:
    """One walk split over lanes: lane t starts at walk index t * keys_per_lane,
    so a hit (t, n) is index t * keys_per_lane + n of the single walk."""
    scal = np.zeros((lanes, 32), np.uint8)
    for t in range(lanes):
        scal[t] = np.frombuffer(step_scalar(start, t * keys_per_lane), np.uint8)
    return WalkSetup(ed_seed, ed25519_public(ed_seed), scal)
