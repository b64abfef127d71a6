"""A tiny interpreter for the integer PTX subset used by the field library's
inline-asm blocks (fe25519_ptx.cuh, fe25519.cuh), so their carry chains can
be checked against Python integers on a machine without a GPU.

Only what the blocks use is implemented: mul/mad/madc (.lo/.hi, with and
without .cc), add/addc, sub/subc (.cc), shf.l.wrap, shl, shr (.u32/.s32),
and, xor, mov, setp (eq, ne, lt, le, gt, ge on .u32), and a predicated
(@p / @!p) bra to a label of the same block.  CC.CF is the carry (or the
borrow, for sub/subc) flag.
"""
from __future__ import annotations

import re

M32 = 0xFFFFFFFF


def _first_colon_outside_strings(asm: str) -> int:
    """Where the template ends: the first ':' not inside a string literal (a
    label inside the template has one of its own)."""
    in_str = False
    i = 0
    while i < len(asm):
        ch = asm[i]
        if in_str and ch == "\\":
            i += 2
            continue
        if ch == '"':
            in_str = not in_str
        elif ch == ":" and not in_str:
            return i
        i += 1
    return len(asm)


def extract_asm_blocks(src: str) -> dict[str, tuple[list[str], int]]:
    """Function name -> (PTX instruction lines, number of outputs)."""
    out = {}
    for m in re.finditer(r"__device__ __forceinline__ (?:void|fe) (\w+)\(([^)]*)\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(3)
        if "asm(" not in body:
            continue
        asm = body[body.index("asm(") :]
        head = asm[: _first_colon_outside_strings(asm)]
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


def run(lines: list[str], args: list[int], branches: dict | None = None) -> list[int]:
    """Execute `lines` with %0.. bound to `args` (outputs first, as zeros).

    `branches`, when given, counts each bra by (label, taken)."""
    regs: dict[str, int] = {}
    preds: dict[str, bool] = {}
    for i, v in enumerate(args):
        regs[f"%{i}"] = v & M32
    cf = 0
    labels = {ln[:-1]: i for i, ln in enumerate(lines) if ln.endswith(":")}

    def val(tok: str) -> int:
        tok = tok.strip()
        if tok in regs:
            return regs[tok]
        if re.fullmatch(r"0[xX][0-9a-fA-F]+|\d+", tok):
            return int(tok, 0) & M32
        raise KeyError(f"undefined operand {tok!r}")

    pc = 0
    while pc < len(lines):
        ln = lines[pc]
        pc += 1
        if ln.endswith(":"):
            continue
        guard = None
        if ln.startswith("@"):
            guard, _, ln = ln.partition(" ")
            neg = guard.startswith("@!")
            guard = preds[guard[2:] if neg else guard[1:]] != neg
        op, _, rest = ln.partition(" ")
        ops = [t.strip() for t in rest.split(",")]
        if op == "bra":
            assert guard is not None, "only predicated branches are used"
            if branches is not None:
                key = (ops[0], guard)
                branches[key] = branches.get(key, 0) + 1
            if guard:
                pc = labels[ops[0]]
            continue
        if guard is not None:
            raise NotImplementedError("predicated " + op)
        parts = op.split(".")
        base = parts[0]
        mods = set(parts[1:])
        if base == "setp":
            x, y = val(ops[1]), val(ops[2])
            assert "u32" in mods, op
            cmp = {"eq": x == y, "ne": x != y, "lt": x < y, "le": x <= y, "gt": x > y, "ge": x >= y}
            preds[ops[0]] = next(v for k, v in cmp.items() if k in mods)
            continue
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
