"""Generates kelvin_horner.cuh: straight-line Horner evaluation of the far-field
polynomial  P(u) = sum_{a+b+c <= lam} coef[g(a,b,c)] ux^a uy^b uz^c  for
lam = 0..8, for 1 and 2 points at a time (sharing every coefficient load).

g() is the degree-graded packing (all monomials of total degree < d first,
then degree d ordered by a, then b), so a coefficient's slot does not depend
on the largest degree in use and one body per lam serves every l_pot_max.
The code is emitted rather than left to template unrolling because nvcc's
optimiser takes tens of minutes on the equivalent nested unrolled loops.

The build (fast_rpa_eval_b200/build.py) writes it into its build directory
before compiling; by hand:

    python gen_kelvin.py <output path>
"""
import os

LMAX = 8


def gidx(a, b, c):
    d = a + b + c
    off = d * (d + 1) * (d + 2) // 6
    pos = 0
    for aa in range(a):
        pos += d - aa + 1
    return off + pos + b


def horner_body(lam, npts):
    out = []
    emit = out.append
    pv = lambda v, j: f"{v}{j}"  # noqa: E731
    first_a = True
    for a in range(lam, -1, -1):
        first_b = True
        for b in range(lam - a, -1, -1):
            top = lam - a - b
            emit(f"    {{ const double k = c[{gidx(a, b, top)}];")
            for j in range(npts):
                emit(f"      double R{j} = k;")
            for cc in range(top - 1, -1, -1):
                emit(f"      {{ const double k2 = c[{gidx(a, b, cc)}];")
                for j in range(npts):
                    emit(f"        R{j} = fma(R{j}, uz[{j}], k2);")
                emit("      }")
            for j in range(npts):
                if first_b:
                    emit(f"      Q{j} = R{j};")
                else:
                    emit(f"      Q{j} = fma(Q{j}, uy[{j}], R{j});")
            emit("    }")
            first_b = False
        for j in range(npts):
            if first_a:
                emit(f"    P[{j}] = Q{j};")
            else:
                emit(f"    P[{j}] = fma(P[{j}], ux[{j}], Q{j});")
        first_a = False
    return "\n".join(out)


def render() -> str:
    lines = [
        "// Generated by gen_kelvin.py: straight-line Horner evaluation of the",
        "// Kelvin-inverted far-field polynomial, degree-graded coefficient packing.",
        "// Do not edit by hand.",
        "#pragma once",
        "",
        "namespace frpa {",
        "",
        f"constexpr int KELVIN_LMAX = {LMAX};",
        "// number of coefficients of degree <= L",
        "__host__ __device__ constexpr int kelvin_count(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }",
        "// slot of ux^a uy^b uz^c",
        "__host__ __device__ constexpr int kelvin_index(int a, int b, int c) {",
        "  return (a + b + c) * (a + b + c + 1) * (a + b + c + 2) / 6 + a * (a + b + c + 1) - a * (a - 1) / 2 + b;",
        "}",
        "",
    ]
    # check the closed form used above against gidx
    for d in range(LMAX + 1):
        for a in range(d + 1):
            for b in range(d - a + 1):
                c = d - a - b
                closed = d * (d + 1) * (d + 2) // 6 + a * (d + 1) - a * (a - 1) // 2 + b
                assert closed == gidx(a, b, c), (a, b, c)
    for npts in (1, 2):
        for lam in range(LMAX + 1):
            lines.append(f"__device__ __forceinline__ void kelvin_horner_{lam}_{npts}(const double *__restrict__ c, "
                         f"const double *ux, const double *uy, const double *uz, double *P) {{")
            lines.append("  " + " ".join(f"double Q{j};" for j in range(npts)))
            lines.append(horner_body(lam, npts))
            lines.append("}")
            lines.append("")
        lines.append(f"__device__ __forceinline__ void kelvin_eval_{npts}(int lam, const double *__restrict__ c, "
                     "const double *ux, const double *uy, const double *uz, double *P) {")
        lines.append("  switch (lam) {")
        for lam in range(LMAX + 1):
            lines.append(f"    case {lam}: kelvin_horner_{lam}_{npts}(c, ux, uy, uz, P); break;")
        lines.append("    default: break;")
        lines.append("  }")
        lines.append("}")
        lines.append("")
    lines.append("// kelvin_eval<N>: N points at a time")
    lines.append("template <int N>")
    lines.append("__device__ __forceinline__ void kelvin_eval(int lam, const double *__restrict__ c, const double *ux, "
                 "const double *uy, const double *uz, double *P);")
    for npts in (1, 2):
        lines.append("template <>")
        lines.append(f"__device__ __forceinline__ void kelvin_eval<{npts}>(int lam, const double *__restrict__ c, "
                     "const double *ux, const double *uy, const double *uz, double *P) {")
        lines.append(f"  kelvin_eval_{npts}(lam, c, ux, uy, uz, P);")
        lines.append("}")
    lines.append("")
    lines.append("}  // namespace frpa")
    lines.append("")
    return "\n".join(lines)


def write(dst: str) -> None:
    text = render()
    if os.path.exists(dst) and open(dst).read() == text:
        return
    with open(dst, "w") as f:
        f.write(text)


if __name__ == "__main__":
    import sys

    write(sys.argv[1])
