"""A tiny interpreter for the integer PTX subset used by the field library's
inline-asm blocks (fe25519_ptx.cuh, fe25519.cuh), so their carry chains can
be checked against Python integers on a machine without a GPU.

Only what the blocks use is implemented: mul/mad/madc (.lo/.hi, with and
without .cc), add/addc, sub/subc (.cc), shf.l.wrap, shl, shr (.u32/.s32),
and, xor, mov.  CC.CF is the carry (or the borrow, for sub/subc) flag.
"""
from __future__ import annotations

import re

M32 = 0xFFFFFFFF


def extract_asm_blocks(src: str) -> dict[str, tuple[list[str], int]]:
    """Function name -> (PTX instruction lines, number of outputs)."""
    out = {}
    for m in re.finditer(r"__device__ __forceinline__ (?:void|fe) (\w+)\(([^)]*)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(3)
        if "asm(" not in body:
            continue
        asm = body[body.index("asm(") :]
        head = asm.split(":")[0]
        strings = re.findall(r'"((?:[^"\\]|\\.)*)"', head)
        text = "".join(strings).replace("\\n", "\n").replace("\\t", " ")
        lines = []
        for ln in text.split("\n"):
            for part in ln.split(";"):
                part = part.strip().strip("{}").strip()
                if part and not part.startswith(".reg"):
                    lines.append(part)
        outs = len(re.findall(r'"=r"', asm))
        out[name] = (lines, outs)
    return out


def run(lines: list[str], args: list[int]) -> list[int]:
    """Execute `lines` with %0.. bound to `args` (outputs first, as zeros)."""
    regs: dict[str, int] = {}
    for i, v in enumerate(args):
        regs[f"%{i}"] = v & M32
    cf = 0

    def val(tok: str) -> int:
        tok = tok.strip()
        if tok in regs:
            return regs[tok]
        if re.fullmatch(r"0[xX][0-9a-fA-F]+|\d+", tok):
            return int(tok, 0) & M32
        raise KeyError(f"undefined operand {tok!r}")

    for ln in lines:
        op, _, rest = ln.partition(" ")
        ops = [t.strip() for t in rest.split(",")]
        parts = op.split(".")
        base = parts[0]
        mods = set(parts[1:])
        cc = "cc" in mods
        d = ops[0]
        if base in ("mul", "mad", "madc"):
            a, b = val(ops[1]), val(ops[2])
            p = a * b
            term = (p >> 32) if "hi" in mods else (p & M32)
            if base == "mul":
                r = term
                regs[d] = r & M32
                continue
            c = val(ops[3])
            r = term + c + (cf if base == "madc" else 0)
        elif base in ("add", "addc"):
            r = val(ops[1]) + val(ops[2]) + (cf if base == "addc" else 0)
        elif base in ("sub", "subc"):
            r = val(ops[1]) - val(ops[2]) - (cf if base == "subc" else 0)
            regs[d] = r & M32
            if cc:
                cf = 1 if r < 0 else 0
            continue
        elif base == "shf":
            lo, hi, n = val(ops[1]), val(ops[2]), val(ops[3]) & 31
            regs[d] = (((hi << 32) | lo) << n >> 32) & M32
            continue
        elif base == "shl":
            regs[d] = (val(ops[1]) << (val(ops[2]) & 31)) & M32
            continue
        elif base == "shr":
            x, n = val(ops[1]), val(ops[2])
            if "s32" in mods and x & 0x80000000:
                x -= 1 << 32
            regs[d] = (x >> n) & M32
            continue
        elif base == "and":
            regs[d] = val(ops[1]) & val(ops[2])
            continue
        elif base == "xor":
            regs[d] = val(ops[1]) ^ val(ops[2])
            continue
        elif base == "mov":
            regs[d] = val(ops[1])
            continue
        else:
            raise NotImplementedError(op)
        regs[d] = r & M32
        if cc:
            cf = r >> 32
            assert cf in (0, 1)
    n_out = sum(1 for k in regs if k.startswith("%"))
    return [regs[f"%{i}"] for i in range(n_out)]


def words(x: int) -> list[int]:
    return [(x >> (32 * i)) & M32 for i in range(8)]


def value(w: list[int]) -> int:
    return sum(v << (32 * i) for i, v in enumerate(w))
