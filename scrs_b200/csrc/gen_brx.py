"""Generate brx_dispatch.cuh: constant multiplication of bit-sliced GF(256)
data through an indirect-branch jump table (PTX brx.idx).

For a coefficient c, multiplying bytes by c is the 8x8 GF(2) matrix
M_c[r][s] = bit r of (c * x^s) over the AES polynomial 0x11B.  On 8 bit planes
p[0..7], acc ^= c*x is acc[r] ^= XOR_{s: M_c[r][s]} p[s].  Each case below is
that XOR network for one c; brx.idx jumps straight to it, so dispatch costs
one indirect branch instead of a compare tree.

    python scrs_b200/csrc/gen_brx.py   (run by scrs_b200/build.py when stale)
"""
from pathlib import Path

OUT = Path(__file__).with_name("brx_dispatch.cuh")


def gf_mul(a, b):
    acc = 0
    for i in range(8):
        if (b >> i) & 1:
            acc ^= a
        hi = a & 0x80
        a = (a << 1) & 0xFF
        if hi:
            a ^= 0x1B
    return acc


def rows_of(c):
    """S_r: the planes XORed into output plane r for coefficient c."""
    cols = [gf_mul(c, 1 << s) for s in range(8)]
    return [[s for s in range(8) if (cols[s] >> r) & 1] for r in range(8)]


def cse_rows(rows):
    """Greedy common-subexpression pass: while some pair of planes occurs in two
    or more rows and sharing it lowers the instruction count, XOR the pair once
    into a temporary and use that in those rows.  Returns (pairs, rows) with
    temporaries numbered 8, 9, ... after the 8 planes."""
    def cost(rs):
        return sum((len(t) + 1) // 2 for t in rs)

    rows = [list(r) for r in rows]
    pairs = []
    while True:
        count = {}
        for r in rows:
            rr = sorted(r)
            for i in range(len(rr)):
                for j in range(i + 1, len(rr)):
                    count[(rr[i], rr[j])] = count.get((rr[i], rr[j]), 0) + 1
        best = None
        for (a, b), n in sorted(count.items()):
            if n < 2:
                continue
            t = 8 + len(pairs)
            new = [[x for x in r if x not in (a, b)] + [t] if (a in r and b in r) else r for r in rows]
            gain = cost(rows) - cost(new) - 1
            if gain > 0 and (best is None or gain > best[0]):
                best = (gain, (a, b), new)
        if best is None:
            return pairs, rows
        pairs.append(best[1])
        rows = best[2]


MAX_TEMPS = 8


def case_body(c, acc_base, p_base, halves, prefix):
    """PTX lines applying coefficient c to `halves` groups of 8 planes: shared
    plane pairs are XORed once into temporaries, then each output plane takes
    its terms two at a time with a 3-input XOR (lop3 0x96)."""
    lines = []
    pairs, rows = cse_rows(rows_of(c))
    assert len(pairs) <= MAX_TEMPS
    for h in range(halves):
        def op(t):
            return f"%{p_base + 8 * h + t}" if t < 8 else f"cse{t - 8}"
        for i, (a, b) in enumerate(pairs):
            lines.append(f"xor.b32 cse{i}, {op(a)}, {op(b)};")
        for r in range(8):
            a = f"%{acc_base + 8 * h + r}"
            terms = list(rows[r])
            while len(terms) >= 2:
                x, y = terms.pop(0), terms.pop(0)
                lines.append(f"lop3.b32 {a}, {a}, {op(x)}, {op(y)}, 0x96;")
            if terms:
                lines.append(f"xor.b32 {a}, {a}, {op(terms[0])};")
    return lines


def dispatch(name, coeffs, halves, acc_base, p_base, idx_op, tag, done, uniform):
    out = []
    labels = [f"{tag}{i}" for i in range(len(coeffs))]
    uni = ".uni" if uniform else ""
    out.append(f"{tag}T: .branchtargets {', '.join(labels)};")
    out.append(f"brx.idx{uni} %{idx_op}, {tag}T;")
    for lab, c in zip(labels, coeffs):
        out.append(f"{lab}:")
        out.extend(case_body(c, acc_base, p_base, halves, tag))
        out.append(f"bra{uni} {done};")
    out.append(f"{done}:")
    return out


def asm_function(fname, doc, nplanes, blocks, uniform=True):
    """blocks: list of (coeff list, index operand name)."""
    halves = nplanes // 8
    n_acc = nplanes
    acc_ops = ", ".join(f'"+r"(a[{i}])' for i in range(n_acc))
    p_ops = ", ".join(f'"r"(p[{i}])' for i in range(nplanes))
    idx_names = [b[1] for b in blocks]
    idx_ops = ", ".join(f'"r"({n})' for n in idx_names)
    body = ["{", f".reg .b32 cse<{MAX_TEMPS}>;"]
    for bi, (coeffs, _) in enumerate(blocks):
        idx_operand = 2 * nplanes + bi
        body += dispatch(fname, coeffs, halves, 0, nplanes, idx_operand, f"L{fname[:2]}{bi}_", f"L{fname[:2]}{bi}_D",
                         uniform)
    body.append("}")
    asm = "\n".join(f'        "{l}\\n"' for l in body)
    params = ", ".join(f"uint32_t {n}" for n in idx_names)
    return f"""// {doc}
__device__ __forceinline__ void {fname}({params}, uint32_t (&a)[{n_acc}], const uint32_t (&p)[{nplanes}]) {{
    asm volatile(
{asm}
        : {acc_ops}
        : {p_ops}, {idx_ops});
}}
"""


def main():
    parts = ["""// Generated by scrs_b200/csrc/gen_brx.py -- do not edit.
// Jump-table constant multiplication of bit-sliced GF(256) planes (see the
// generator for the construction).  Labels live inside a PTX { } scope, so
// each inlined copy has its own.
#pragma once
#include <stdint.h>

namespace scrs {
"""]
    parts.append(asm_function("brx_mul8x2_nib",
                              "Both tower components: acc[0..7] ^= v*p[0..7], acc[8..15] ^= v*p[8..15], "
                              "v = lo + 16*hi.", 16,
                              [(list(range(16)), "lo"), ([v << 4 for v in range(16)], "hi")]))
    parts.append(asm_function("brx_mul8x2_lo",
                              "acc[0..7] ^= v*p[0..7], acc[8..15] ^= v*p[8..15] for v < 16: one 16-way jump.", 16,
                              [(list(range(16)), "v")]))
    parts.append(asm_function("brx_mul8x2_nib_div",
                              "As brx_mul8x2_nib, for coefficients that may differ across the warp.", 16,
                              [(list(range(16)), "lo"), ([v << 4 for v in range(16)], "hi")], uniform=False))
    parts.append("}  // namespace scrs\n")
    OUT.write_text("\n".join(parts))


if __name__ == "__main__":
    main()
