#!/usr/bin/env python3
"""Generates fe25519_ptx.cuh: GF(2^255-19) multiply and square on 8 x 32-bit
limbs as single inline-PTX blocks, so that each carry chain stays inside one
asm statement (the carry flag is not preserved between asm statements).

Representation: a field element is any 256-bit value x (8 little-endian
32-bit words) standing for x mod p, p = 2^255 - 19.  Products are reduced
with 2^256 = 38 (mod p) to another 256-bit value; only fe_canon (in
fe25519.cuh) maps to [0, p).

Run from this directory: python gen_fe_ptx.py > fe25519_ptx.cuh
"""


def mul_body(square: bool) -> list[str]:
    """PTX lines computing r0..r15 = a * b (or a * a), then the reduction
    into %0..%7.  Inputs are %8..%15 (a) and %16..%23 (b)."""
    A = [f"%{8 + i}" for i in range(8)]
    B = A if square else [f"%{16 + i}" for i in range(8)]
    L = []
    L.append(".reg .u32 r<16>;")
    L.append(".reg .u32 c, c2, t;")
    L.append(".reg .pred p;")
    if not square:
        # Row 0: r[0..8] = a0 * b.
        L.append(f"mul.lo.u32 r0, {A[0]}, {B[0]};")
        for j in range(1, 8):
            L.append(f"mul.lo.u32 r{j}, {A[0]}, {B[j]};")
        L.append(f"mul.hi.u32 r8, {A[0]}, {B[7]};")
        # hi parts of row 0 into r1..r8
        L.append(f"mad.hi.cc.u32 r1, {A[0]}, {B[0]}, r1;")
        for j in range(1, 7):
            L.append(f"madc.hi.cc.u32 r{j + 1}, {A[0]}, {B[j]}, r{j + 1};")
        L.append("addc.u32 r8, r8, 0;")
        # Rows 1..7.
        for i in range(1, 8):
            # lo parts: r[i+j] += lo(a_i b_j), carry into r[i+8]
            L.append(f"mad.lo.cc.u32 r{i}, {A[i]}, {B[0]}, r{i};")
            for j in range(1, 8):
                L.append(f"madc.lo.cc.u32 r{i + j}, {A[i]}, {B[j]}, r{i + j};")
            if i + 8 <= 15:
                if i == 1:
                    L.append(f"addc.u32 r{i + 8}, 0, 0;")
                else:
                    L.append(f"addc.u32 r{i + 8}, r{i + 8}, 0;")
            # hi parts: r[i+j+1] += hi(a_i b_j), carry into r[i+9]
            L.append(f"mad.hi.cc.u32 r{i + 1}, {A[i]}, {B[0]}, r{i + 1};")
            for j in range(1, 8):
                L.append(f"madc.hi.cc.u32 r{i + j + 1}, {A[i]}, {B[j]}, r{i + j + 1};")
            if i + 9 <= 15:
                L.append(f"addc.u32 r{i + 9}, 0, 0;")
    else:
        # Cross products a_i a_j (i < j) into r1..r14, then double, then add
        # the squares a_i^2 at r[2i], r[2i+1].
        # Row 0: r[1..8] = a0 * a[1..7]
        for j in range(1, 8):
            L.append(f"mul.lo.u32 r{j}, {A[0]}, {A[j]};")
        L.append(f"mul.hi.u32 r8, {A[0]}, {A[7]};")
        L.append(f"mad.hi.cc.u32 r2, {A[0]}, {A[1]}, r2;")
        for j in range(2, 7):
            L.append(f"madc.hi.cc.u32 r{j + 1}, {A[0]}, {A[j]}, r{j + 1};")
        L.append("addc.u32 r8, r8, 0;")
        # Row i (1..6): r[2i+1 .. i+8] += a_i * a[i+1..7]
        for i in range(1, 7):
            js = list(range(i + 1, 8))
            first = True
            for j in js:
                op = "mad.lo.cc.u32" if first else "madc.lo.cc.u32"
                L.append(f"{op} r{i + j}, {A[i]}, {A[j]}, r{i + j};")
                first = False
            top = i + 8
            if i == 1:
                L.append(f"addc.u32 r{top}, 0, 0;")
            else:
                L.append(f"addc.u32 r{top}, r{top}, 0;")
            first = True
            for j in js:
                op = "mad.hi.cc.u32" if first else "madc.hi.cc.u32"
                L.append(f"{op} r{i + j + 1}, {A[i]}, {A[j]}, r{i + j + 1};")
                first = False
            if top + 1 <= 15:
                L.append(f"addc.u32 r{top + 1}, 0, 0;")
        # r0 = 0 so far.  The cross sum is below 2^511, so doubling r1..r15
        # in place (high word first) loses nothing.
        for k in range(15, 1, -1):
            L.append(f"shf.l.wrap.b32 r{k}, r{k - 1}, r{k}, 1;")
        L.append("shl.b32 r1, r1, 1;")
        # Add the squares.
        L.append(f"mul.lo.u32 r0, {A[0]}, {A[0]};")
        L.append(f"mad.hi.cc.u32 r1, {A[0]}, {A[0]}, r1;")
        for i in range(1, 8):
            L.append(f"madc.lo.cc.u32 r{2 * i}, {A[i]}, {A[i]}, r{2 * i};")
            if i < 7:
                L.append(f"madc.hi.cc.u32 r{2 * i + 1}, {A[i]}, {A[i]}, r{2 * i + 1};")
            else:
                L.append(f"madc.hi.u32 r15, {A[i]}, {A[i]}, r15;")
    L.extend(reduce_lines())
    return L


def reduce_lines() -> list[str]:
    """r0..r15 (512 bits) -> %0..%7 with 2^256 = 38; result < 2^256."""
    L = []
    # lo parts: r[k] += lo(38 r[k+8]); carry into c.
    L.append("mad.lo.cc.u32 r0, r8, 38, r0;")
    for k in range(1, 8):
        L.append(f"madc.lo.cc.u32 r{k}, r{k + 8}, 38, r{k};")
    L.append("addc.u32 c, 0, 0;")
    # hi parts: r[k+1] += hi(38 r[k+8]); top into c.
    L.append("mad.hi.cc.u32 r1, r8, 38, r1;")
    for k in range(1, 7):
        L.append(f"madc.hi.cc.u32 r{k + 1}, r{k + 8}, 38, r{k + 1};")
    L.append("madc.hi.u32 c, r15, 38, c;")
    # value = r0..r7 + c 2^256 with c <= 38: fold c once more.  The add into
    # r0 carries into r1 with probability below 2^-21, so that chain is a
    # branch the common case skips.
    L.append("mul.lo.u32 t, c, 38;")
    L.append("add.cc.u32 r0, r0, t;")
    L.append("addc.u32 c2, 0, 0;")
    L.append("setp.eq.u32 p, c2, 0;")
    L.append("@p bra FOLDED;")
    L.append("add.cc.u32 r1, r1, 1;")
    for k in range(2, 8):
        L.append(f"addc.cc.u32 r{k}, r{k}, 0;")
    L.append("addc.u32 c2, 0, 0;")
    # A carry here leaves r0..r7 < 38 * 39: adding 38 cannot carry.
    L.append("mad.lo.u32 r0, c2, 38, r0;")
    L.append("FOLDED:")
    for k in range(8):
        L.append(f"mov.u32 %{k}, r{k};")
    return L


def emit_asm(name: str, lines: list[str], square: bool) -> str:
    out = []
    params = "fe& o, const fe& a" if square else "fe& o, const fe& a, const fe& b"
    out.append(f"__device__ __forceinline__ void {name}({params}) {{")
    out.append("    asm(\"{\\n\\t\"")
    for ln in lines:
        out.append(f"        \"{ln}\\n\\t\"")
    out.append("        \"}\"")
    outs = ", ".join(f'"=r"(o.v[{i}])' for i in range(8))
    ins_a = ", ".join(f'"r"(a.v[{i}])' for i in range(8))
    if square:
        out.append(f"        : {outs}")
        out.append(f"        : {ins_a});")
    else:
        ins_b = ", ".join(f'"r"(b.v[{i}])' for i in range(8))
        out.append(f"        : {outs}")
        out.append(f"        : {ins_a},")
        out.append(f"          {ins_b});")
    out.append("}")
    return "\n".join(out)


def main() -> None:
    print("// Generated by gen_fe_ptx.py: do not edit by hand.")
    print("// 8 x 32-bit limb multiply and square mod 2^255-19 (2^256 = 38), one")
    print("// inline-PTX block each so every carry chain stays in one asm statement.")
    print("#pragma once")
    print()
    print(emit_asm("fe_mul_ptx", mul_body(False), False))
    print()
    print(emit_asm("fe_sqr_ptx", mul_body(True), True))


if __name__ == "__main__":
    main()
