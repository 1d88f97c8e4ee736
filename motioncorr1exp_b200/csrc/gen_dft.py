"""Generate dft_gen.cuh: straight-line radix-R DFT butterflies.

Odd radices use the symmetric form of a direct DFT: with s_n = x_n + x_{R-n}
and d_n = x_n - x_{R-n} (n = 1..h, h = (R-1)/2),

    X_0     = x_0 + sum_n s_n
    A_k     = x_0 + sum_n s_n cos(2 pi n k / R)
    B_k     = sum_n d_n sin(2 pi n k / R)
    X_k     = A_k -/+ i B_k,   X_{R-k} = A_k +/- i B_k      (forward / inverse)

which costs 4 h^2 FMAs instead of 4 R^2.  The cosines and sines are emitted as
float literals (rounded once from float64), so the compiler folds them into
the FMA instructions.  Run:  python gen_dft.py > dft_gen.cuh
"""
import math
import sys

ODD_RADICES = [3, 5, 7, 11, 13, 53]


def flit(x: float) -> str:
    v = float(__import__("numpy").float32(x))
    if v == 0.0:
        return "0.0f"
    return repr(v) + "f"


def emit_odd(R: int) -> str:
    h = (R - 1) // 2
    L = []
    L.append(f"template <bool INV> __device__ __forceinline__ void dft_r{R}(float2* v) {{")
    L.append("  const float2 x0 = v[0];")
    for n in range(1, h + 1):
        L.append(f"  const float2 s{n} = make_float2(v[{n}].x + v[{R-n}].x, v[{n}].y + v[{R-n}].y);")
        L.append(f"  const float2 d{n} = make_float2(v[{n}].x - v[{R-n}].x, v[{n}].y - v[{R-n}].y);")
    sx = " + ".join([f"s{n}.x" for n in range(1, h + 1)])
    sy = " + ".join([f"s{n}.y" for n in range(1, h + 1)])
    L.append(f"  v[0] = make_float2(x0.x + ({sx}), x0.y + ({sy}));")
    for k in range(1, h + 1):
        L.append("  {")
        L.append("    float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;")
        for n in range(1, h + 1):
            m = (n * k) % R
            c = flit(math.cos(2.0 * math.pi * m / R))
            s = flit(math.sin(2.0 * math.pi * m / R))
            L.append(f"    ar = fmaf(s{n}.x, {c}, ar); ai = fmaf(s{n}.y, {c}, ai);"
                     f" br = fmaf(d{n}.x, {s}, br); bi = fmaf(d{n}.y, {s}, bi);")
        # forward: X_k = A - iB = (ar + bi, ai - br); X_{R-k} = (ar - bi, ai + br)
        L.append("    if (!INV) {")
        L.append(f"      v[{k}] = make_float2(ar + bi, ai - br); v[{R-k}] = make_float2(ar - bi, ai + br);")
        L.append("    } else {")
        L.append(f"      v[{k}] = make_float2(ar - bi, ai + br); v[{R-k}] = make_float2(ar + bi, ai - br);")
        L.append("    }")
        L.append("  }")
    L.append("}")
    return "\n".join(L)


def main() -> None:
    out = []
    out.append("// Generated by gen_dft.py -- do not edit by hand.")
    out.append("// Straight-line odd-radix DFT butterflies (symmetric direct form).")
    out.append("#pragma once")
    out.append("#include <cuda_runtime.h>")
    out.append("namespace mc {")
    out.append(f"constexpr int kGeneratedOddRadices[] = {{{', '.join(map(str, ODD_RADICES))}}};")
    for R in ODD_RADICES:
        out.append(emit_odd(R))
    out.append("}  // namespace mc")
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
