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
    if R < 53:
        # MC_PACKED_FMA=1: the cosine and sine sums on packed FP32 pairs, one
        # fma.f32x2 per term for the real and imaginary halves
        L.append("#if MC_PACKED_FMA")
        for n in range(1, h + 1):
            L.append(f"  const f2reg S{n} = f2pk(padd(v[{n}], v[{R-n}]));")
            L.append(f"  const f2reg D{n} = f2pk(psub(v[{n}], v[{R-n}]));")
        sx = " + ".join([f"v[{n}].x + v[{R-n}].x" for n in range(1, h + 1)])
        sy = " + ".join([f"v[{n}].y + v[{R-n}].y" for n in range(1, h + 1)])
        L.append(f"  {{ float2 t = f2up(S1);")
        for n in range(2, h + 1):
            L.append(f"    {{ const float2 u = f2up(S{n}); t.x += u.x; t.y += u.y; }}")
        L.append("    v[0] = make_float2(x0.x + t.x, x0.y + t.y); }")
        for k in range(1, h + 1):
            L.append("  {")
            L.append("    f2reg A = f2pk(x0), B = 0ull;")
            for n in range(1, h + 1):
                m = (n * k) % R
                c = flit(math.cos(2.0 * math.pi * m / R))
                s = flit(math.sin(2.0 * math.pi * m / R))
                L.append(f"    A = f2fma(S{n}, f2splat({c}), A); B = f2fma(D{n}, f2splat({s}), B);")
            L.append("    const float2 a = f2up(A), b = f2up(B);")
            L.append("    if (!INV) {")
            L.append(f"      v[{k}] = make_float2(a.x + b.y, a.y - b.x); v[{R-k}] = make_float2(a.x - b.y, a.y + b.x);")
            L.append("    } else {")
            L.append(f"      v[{k}] = make_float2(a.x - b.y, a.y + b.x); v[{R-k}] = make_float2(a.x + b.y, a.y - b.x);")
            L.append("    }")
            L.append("  }")
        L.append("#else")
    for n in range(1, h + 1):
        L.append(f"  const float2 s{n} = padd(v[{n}], v[{R-n}]);")
        L.append(f"  const float2 d{n} = psub(v[{n}], v[{R-n}]);")
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
    if R < 53:
        L.append("#endif")
    L.append("}")
    return "\n".join(L)


def emit_odd_split(R: int, S: int) -> str:
    """Radix-R butterfly whose outputs are split over S threads: part p
    computes X_0 (p == 0) and the pairs (X_k, X_{R-k}) of its k-range, and
    hands each output to st(index, value)."""
    h = (R - 1) // 2
    bounds = [round(i * h / S) for i in range(S + 1)]
    L = [f"template <bool INV, typename St>",
         f"__device__ __forceinline__ void dft_r{R}_part(const float2* v, int part, St&& st) {{",
         "  const float2 x0 = v[0];"]
    for n in range(1, h + 1):
        L.append(f"  const float2 s{n} = padd(v[{n}], v[{R-n}]);")
        L.append(f"  const float2 d{n} = psub(v[{n}], v[{R-n}]);")
    sx = " + ".join([f"s{n}.x" for n in range(1, h + 1)])
    sy = " + ".join([f"s{n}.y" for n in range(1, h + 1)])
    L.append(f"  if (part == 0) st(0, make_float2(x0.x + ({sx}), x0.y + ({sy})));")
    L.append("  switch (part) {")
    for p in range(S):
        L.append(f"  case {p}: {{")
        for k in range(bounds[p] + 1, bounds[p + 1] + 1):
            L.append("    {")
            L.append("      float ar = x0.x, ai = x0.y, br = 0.0f, bi = 0.0f;")
            for n in range(1, h + 1):
                m = (n * k) % R
                c = flit(math.cos(2.0 * math.pi * m / R))
                s = flit(math.sin(2.0 * math.pi * m / R))
                L.append(f"      ar = fmaf(s{n}.x, {c}, ar); ai = fmaf(s{n}.y, {c}, ai);"
                         f" br = fmaf(d{n}.x, {s}, br); bi = fmaf(d{n}.y, {s}, bi);")
            L.append(f"      if (!INV) {{ st({k}, make_float2(ar + bi, ai - br)); st({R-k}, make_float2(ar - bi, ai + br)); }}")
            L.append(f"      else {{ st({k}, make_float2(ar - bi, ai + br)); st({R-k}, make_float2(ar + bi, ai - br)); }}")
            L.append("    }")
        L.append("    break;")
        L.append("  }")
    L.append("  default: break;")
    L.append("  }")
    L.append("}")
    return "\n".join(L)


def emit_odd_compact(R: int) -> str:
    """Radix-R DFT with a runtime loop over the (R-1)/2 output pairs: the
    pairs' twiddles come from a __constant__ table (uniform index, broadcast),
    so the code is ~h times smaller than the straight-line form; each output
    goes to st(index, value) as soon as it is formed.  The sums run on packed
    FP32 pairs (one fma.f32x2 per term for the real and imaginary halves,
    each rounded as the scalar FMA).  PAIRED = true forms two output pairs
    (k, k + h/2) per iteration (twice the independent chains).  Without
    PAIRED only the output pairs (k, R - k) with k <= kmax are formed (X_0
    always): a pruned transform whose other outputs are not wanted."""
    h = (R - 1) // 2
    rows = []
    for k in range(h + 1):
        row = []
        for n in range(h + 1):
            m = (n * k) % R
            row.append(f"{{{flit(math.cos(2 * math.pi * m / R))}, {flit(math.sin(2 * math.pi * m / R))}}}")
        rows.append("{" + ", ".join(row) + "}")
    L = [f"__constant__ float2 c_tw{R}[{h + 1}][{h + 1}] = {{" + ",\n  ".join(rows) + "};",
         f"template <bool INV, bool PAIRED = false, typename St>",
         f"__device__ __forceinline__ void dft_r{R}_compact(const float2* v, St&& st, int kmax = {h}) {{",
         "  const float2 x0 = v[0];",
         "  const f2reg X0 = f2pk(x0);"]
    for n in range(1, h + 1):
        L.append(f"  const f2reg S{n} = f2add(f2pk(v[{n}]), f2pk(v[{R-n}]));")
        L.append(f"  const f2reg D{n} = f2sub(f2pk(v[{n}]), f2pk(v[{R-n}]));")
    L.append("  {")
    L.append("    f2reg t = S1;")
    for n in range(2, h + 1):
        L.append(f"    t = f2add(t, S{n});")
    L.append("    st(0, f2up(f2add(X0, t)));")
    L.append("  }")

    def emit_out(kexpr, A, B, indent):
        return [f"{indent}{{ const float2 a = f2up({A}), b = f2up({B});",
                f"{indent}  if (!INV) {{ st({kexpr}, make_float2(a.x + b.y, a.y - b.x));"
                f" st({R} - ({kexpr}), make_float2(a.x - b.y, a.y + b.x)); }}",
                f"{indent}  else {{ st({kexpr}, make_float2(a.x - b.y, a.y + b.x));"
                f" st({R} - ({kexpr}), make_float2(a.x + b.y, a.y - b.x)); }} }}"]

    def single(kexpr, indent):
        out = [f"{indent}const float2* t = c_tw{R}[{kexpr}];",
               f"{indent}f2reg A = X0, B = 0ull;"]
        for n in range(1, h + 1):
            out.append(f"{indent}{{ const float2 c = t[{n}]; A = f2fma(S{n}, f2splat(c.x), A);"
                       f" B = f2fma(D{n}, f2splat(c.y), B); }}")
        out += emit_out(kexpr, "A", "B", indent)
        return out

    half = h // 2
    L.append("  if constexpr (PAIRED) {")
    L.append("#pragma unroll 1")
    L.append(f"    for (int k = 1; k <= {half}; k++) {{")
    L.append(f"      const float2* t = c_tw{R}[k];")
    L.append(f"      const float2* u = c_tw{R}[k + {half}];")
    L.append("      f2reg A = X0, B = 0ull, C = X0, E = 0ull;")
    for n in range(1, h + 1):
        L.append(f"      {{ const float2 c = t[{n}], e = u[{n}];"
                 f" A = f2fma(S{n}, f2splat(c.x), A); B = f2fma(D{n}, f2splat(c.y), B);"
                 f" C = f2fma(S{n}, f2splat(e.x), C); E = f2fma(D{n}, f2splat(e.y), E); }}")
    L += emit_out("k", "A", "B", "      ")
    L += emit_out(f"k + {half}", "C", "E", "      ")
    L.append("    }")
    if h % 2:
        L.append("    {")
        L += single(str(h), "      ")
        L.append("    }")
    L.append("  } else {")
    L.append("#pragma unroll 1")
    L.append(f"    for (int k = 1; k <= kmax; k++) {{")
    L += single("k", "      ")
    L.append("    }")
    L.append("  }")
    L.append("}")
    return "\n".join(L)


def factor_codelet(q: int) -> list:
    """Radix order used for register codelets: odd radices first, then 8/4/2."""
    rad, m = [], q
    for p in (7, 5, 3):
        while m % p == 0:
            rad.append(p)
            m //= p
    twos = 0
    while m % 2 == 0:
        twos += 1
        m //= 2
    if m != 1:
        raise ValueError(f"{q} has a factor outside 2,3,5,7")
    pw = []
    while twos >= 3:
        if twos == 4:
            pw += [4, 4]
            twos = 0
            break
        pw.append(8)
        twos -= 3
    if twos == 2:
        pw.append(4)
    if twos == 1:
        pw.append(2)
    return rad + pw


# Radices the prime-factor codelets combine (dft_any handles each).
PFA_RADICES = (2, 3, 4, 5, 7, 8)


def pfa_plan(q: int):
    """Good-Thomas prime-factor plan of length q: its prime-power groups when
    there are at least two and each is a radix dft_any handles, else None.
    Returns (groups, input multipliers M_i = q / g_i, CRT factors t_i =
    M_i^-1 mod g_i).  With n = sum n_i M_i and k = sum k_i M_i t_i (mod q),
    W_q^(n k) = prod W_(g_i)^(n_i k_i): the transform is a product of
    independent g_i-point DFTs with no twiddle factors between them."""
    groups, m, p = [], q, 2
    while m > 1:
        if m % p == 0:
            g = 1
            while m % p == 0:
                g *= p
                m //= p
            groups.append(g)
        p += 1
    if len(groups) < 2 or any(g not in PFA_RADICES for g in groups):
        return None
    M = [q // g for g in groups]
    t = [pow(M[i] % groups[i], -1, groups[i]) for i in range(len(groups))]
    return groups, M, t


def pfa_indices(q: int):
    """(input index, output index) of every multi-index of the PFA plan, in
    the working array's order (multi-index (n_0, n_1, ...) at
    n_0 + g_0 (n_1 + g_1 (...)))."""
    groups, M, t = pfa_plan(q)
    import itertools
    ins, outs = [], []
    for idx in itertools.product(*[range(g) for g in reversed(groups)]):
        nidx = list(reversed(idx))
        ins.append(sum(n * Mi for n, Mi in zip(nidx, M)) % q)
        outs.append(sum(k * Mi * ti for k, Mi, ti in zip(nidx, M, t)) % q)
    return groups, ins, outs


def emit_codelet_pfa(q: int) -> str:
    """In-register prime-factor (Good-Thomas) FFT of length q: the input
    gathered by the Ruritanian map, small DFTs along each group's axis with
    no twiddles, the output scattered by the CRT map."""
    groups, ins, outs = pfa_indices(q)
    G = len(groups)
    strides = [1] * G
    for d in range(1, G):
        strides[d] = strides[d - 1] * groups[d - 1]
    L = [f"template <bool INV> __device__ __forceinline__ void fft_pfa_{q}(float2* a) {{",
         f"  // prime-factor plan {' x '.join(map(str, groups))}: no twiddle factors",
         f"  float2 b[{q}];"]
    for w in range(q):
        L.append(f"  b[{w}] = a[{ins[w]}];")
    for d in range(G):
        g, st = groups[d], strides[d]
        for base in range(q):
            if (base // st) % g:
                continue
            L.append("  {")
            L.append(f"    float2 x[{g}];")
            for r in range(g):
                L.append(f"    x[{r}] = b[{base + r * st}];")
            L.append(f"    dft_any<{g}, INV>(x);")
            for r in range(g):
                L.append(f"    b[{base + r * st}] = x[{r}];")
            L.append("  }")
    for w in range(q):
        L.append(f"  a[{outs[w]}] = b[{w}];")
    L.append("}")
    return "\n".join(L)


def emit_codelet(q: int) -> str:
    """In-register Stockham FFT of length q with every index and twiddle
    resolved at generation time: fft_reg_q<INV>(float2 a[q]), result in a."""
    radices = factor_codelet(q)
    L = [f"template <bool INV> __device__ __forceinline__ void fft_reg_{q}(float2* a) {{",
         f"  float2 b[{q}];"]
    ns, src, dst = 1, "a", "b"
    for R in radices:
        nq = q // R
        for j in range(nq):
            jm, jq = j % ns, j // ns
            L.append("  {")
            L.append(f"    float2 x[{R}];")
            for r in range(R):
                L.append(f"    x[{r}] = {src}[{j + r * nq}];")
            if ns > 1:
                for r in range(1, R):
                    e = (r * jm * (q // (ns * R))) % q
                    if e == 0:
                        continue
                    if 4 * e == q:
                        L.append(f"    x[{r}] = rot90<INV>(x[{r}]);")
                        continue
                    if 2 * e == q:
                        L.append(f"    x[{r}] = make_float2(-x[{r}].x, -x[{r}].y);")
                        continue
                    if 4 * e == 3 * q:
                        L.append(f"    x[{r}] = rot90<!INV>(x[{r}]);")
                        continue
                    c = flit(math.cos(2.0 * math.pi * e / q))
                    s = flit(-math.sin(2.0 * math.pi * e / q))
                    L.append(f"    x[{r}] = cmul(x[{r}], make_float2({c}, INV ? -({s}) : ({s})));")
            L.append(f"    dft_any<{R}, INV>(x);")
            base = jq * ns * R + jm
            for r in range(R):
                L.append(f"    {dst}[{base + r * ns}] = x[{r}];")
            L.append("  }")
        src, dst = dst, src
        ns *= R
    if src != "a":
        L.append(f"#pragma unroll\n  for (int i = 0; i < {q}; i++) a[i] = b[i];")
    L.append("}")
    return "\n".join(L)


CODELETS = [4, 8, 10, 12, 14, 16, 20, 24, 28, 30, 32, 35, 40, 48, 56, 60, 64, 70]
SPLIT53 = 3


def main() -> None:
    which = sys.argv[1] if len(sys.argv) > 1 else "dft"
    out = []
    out.append("// Generated by gen_dft.py -- do not edit by hand.")
    if which == "dft":
        out.append("// Straight-line odd-radix DFT butterflies (symmetric direct form).")
        out.append("#pragma once")
        out.append("#include <cuda_runtime.h>")
        out.append('#include "f2ops.cuh"')
        out.append("// MC_PACKED_FMA=1: the odd butterflies' sums on packed FP32 pairs (bitwise")
        out.append("// the same results: each half is the scalar FMA chain)")
        out.append("#ifndef MC_PACKED_FMA")
        out.append("#define MC_PACKED_FMA 0")
        out.append("#endif")
        out.append("namespace mc {")
        out.append(f"constexpr int kGeneratedOddRadices[] = {{{', '.join(map(str, ODD_RADICES))}}};")
        for R in ODD_RADICES:
            out.append(emit_odd(R))
        out.append(f"constexpr int kSplit53 = {SPLIT53};")
        out.append(emit_odd_split(53, SPLIT53))
        out.append(emit_odd_compact(53))
        out.append("}  // namespace mc")
    else:
        out.append("// Register-resident FFT codelets (lengths with factors 2, 3, 5, 7).")
        out.append("#pragma once")
        out.append('#include "fft_engine.cuh"')
        out.append("namespace mc {")
        out.append(f"constexpr int kCodelets[] = {{{', '.join(map(str, CODELETS))}}};")
        out.append(f"constexpr int kNumCodelets = {len(CODELETS)};")
        for q in CODELETS:
            out.append(emit_codelet(q))
        out.append("template <int Q, bool INV> __device__ __forceinline__ void fft_reg(float2* a) {")
        for i, q in enumerate(CODELETS):
            kw = "if" if i == 0 else "else if"
            out.append(f"  {kw} constexpr (Q == {q}) fft_reg_{q}<INV>(a);")
        out.append("}")
        # prime-factor (Good-Thomas) forms of the lengths with coprime factors:
        # the pair kernels use them (measured faster there; the forward
        # transforms keep the Stockham forms, which measured faster in them)
        for q in CODELETS:
            if pfa_plan(q):
                out.append(emit_codelet_pfa(q))
        out.append("template <int Q, bool INV> __device__ __forceinline__ void fft_reg_pf(float2* a) {")
        first = True
        for q in CODELETS:
            if pfa_plan(q):
                out.append(f"  {'if' if first else 'else if'} constexpr (Q == {q}) fft_pfa_{q}<INV>(a);")
                first = False
        out.append("  else fft_reg<Q, INV>(a);")
        out.append("}")
        out.append("}  // namespace mc")
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
