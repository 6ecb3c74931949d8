"""Generate legendre_tables.cuh: constants of the normalised Legendre recurrence.

Agama's normalisation (the one the reference's kernels use,
_multipole_potential_kernel.cu:44-94): Y_lm = N_lm P_l^m(cos theta) with
N_lm = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!), P_l^m including the Condon-Shortley
phase, times 2 sqrt(pi) (m = 0) or 2 sqrt(2 pi) (m != 0).

Instead of the reference's un-normalised recurrence with a sqrt per (l,|m|)
step, the kernels run the recurrence directly on Ybar_l^m = mul_m N_lm P_l^m:

    Ybar_m^m     = SEED[m] sin^m(theta),   SEED[m] = mul_m N_mm (-1)^m (2m-1)!!
    Ybar_l^m     = ALPHA[m][l] (cos(theta) Ybar_{l-1}^m) - BETA[m][l] Ybar_{l-2}^m
    ALPHA[m][l]  = sqrt((4l^2 - 1) / (l^2 - m^2))
    BETA[m][l]   = sqrt((2l+1) ((l-1)^2 - m^2) / ((2l-3) (l^2 - m^2)))

All constants are evaluated in 50-digit decimal arithmetic and rounded once,
except the m != 0 angular factor: the reference hard-codes it as
5.0132565706694072 (_multipole_potential_kernel.cu:94, _cylspl_potential_kernel.cu:67,
gpu_potential.py:962), which is 2 sqrt(2 pi) * (1 + 4.27e-9).  Every m != 0
term of the reference carries that factor, so the kernels use the same literal
to reproduce its results.
"""
from decimal import Decimal, getcontext
from math import factorial
from pathlib import Path

getcontext().prec = 50
LMAX = 32
PI = Decimal("3.14159265358979323846264338327950288419716939937510")


def dsqrt(x: Decimal) -> Decimal:
    return x.sqrt()


def prefact(m: int) -> Decimal:
    return dsqrt(Decimal(2 * m + 1) / (4 * PI * Decimal(factorial(2 * m))))


def dfact_odd(m: int) -> int:          # (2m-1)!!
    out = 1
    for k in range(1, 2 * m, 2):
        out *= k
    return out


def main(out_path: Path) -> None:
    mul0 = 2 * dsqrt(PI)
    mul1 = Decimal("5.0132565706694072")      # reference literal, see module docstring
    seed, pref, coef = [], [], []
    for m in range(LMAX + 1):
        p = prefact(m)
        c = (-1) ** m * dfact_odd(m) * p
        pref.append(p)
        coef.append(c)
        seed.append((mul0 if m == 0 else mul1) * c)
    norm = []
    for m in range(LMAX + 1):
        for l in range(LMAX + 1):
            norm.append(dsqrt(Decimal(2 * l + 1) / (4 * PI) * Decimal(factorial(l - m)) /
                              Decimal(factorial(l + m))) if l >= m else Decimal(0))
    alpha = []
    beta = []
    for m in range(LMAX + 1):
        for l in range(LMAX + 1):
            if l <= m:
                alpha.append(Decimal(0))
                beta.append(Decimal(0))
                continue
            den = Decimal(l * l - m * m)
            alpha.append(dsqrt(Decimal(4 * l * l - 1) / den))
            if l >= m + 2:
                beta.append(dsqrt(Decimal((2 * l + 1) * ((l - 1) ** 2 - m * m)) /
                                  (Decimal(2 * l - 3) * den)))
            else:
                beta.append(Decimal(0))

    # Rescaled recurrence Q_l = Ybar_l / C_l with C_l = prod_{j=m+1..l} ALPHA[m][j]:
    #   Q_l = cos(theta) Q_{l-1} - BETAQ[m][l] Q_{l-2},  BETAQ = BETA[m][l] / (ALPHA[m][l] ALPHA[m][l-1])
    # (stored negated); the C_l are folded into the coefficient tables of regular
    # structures, so the walk needs one constant and one multiply less per step.
    nbetaq = []
    for m in range(LMAX + 1):
        for l in range(LMAX + 1):
            i = m * (LMAX + 1) + l
            if l >= m + 2:
                nbetaq.append(-beta[i] / (alpha[i] * alpha[i - 1]))
            else:
                nbetaq.append(Decimal(0))

    # Two-step form for even-l (symmetric) walks: from Q_l = c Q_{l-1} + NB_l Q_{l-2}
    # applied at l and l-1 and c Q_{l-3} = Q_{l-2} - NB_{l-2} Q_{l-4},
    #   Q_l = (c^2 + SKIPA[m][l]) Q_{l-2} + SKIPB[m][l] Q_{l-4}
    #   SKIPA = NB_l + NB_{l-1},  SKIPB = -NB_{l-1} NB_{l-2}
    # (NB = NBETAQ, zero below l = m + 2, which makes the first step of every
    # walk exact).  Stored for even l only, index m * 17 + l / 2, as (A, B) pairs.
    def nb(m, l):
        return nbetaq[m * (LMAX + 1) + l] if 0 <= l <= LMAX else Decimal(0)
    skip = []
    for m in range(LMAX + 1):
        for j in range(LMAX // 2 + 1):
            l = 2 * j
            if l >= m + 2:
                skip.append((nb(m, l) + nb(m, l - 1), -nb(m, l - 1) * nb(m, l - 2)))
            else:
                skip.append((Decimal(0), Decimal(0)))

    def arr2(name, pairs, typ="double2", suffix=""):
        items = [f"{{{float(a)!r}{suffix}, {float(b)!r}{suffix}}}" for a, b in pairs]
        lines = [", ".join(items[i:i + 2]) for i in range(0, len(items), 2)]
        return (f"__constant__ {typ} {name}[{len(pairs)}] = {{\n    " +
                ",\n    ".join(lines) + "\n};\n")

    def arr(name, vals, typ="double", per_line=4):
        items = [f"{float(v)!r}" + ("f" if typ == "float" else "") for v in vals]
        lines = [", ".join(items[i:i + per_line]) for i in range(0, len(items), per_line)]
        return (f"__constant__ {typ} {name}[{len(vals)}] = {{\n    " +
                ",\n    ".join(lines) + "\n};\n")

    src = ["// Generated by gen_tables.py -- do not edit.",
           "// Constants of the normalised associated-Legendre recurrence (Agama normalisation).",
           "#pragma once",
           f"#define AGB_LEG_N {LMAX + 1}",
           f"#define AGB_MUL0 {float(mul0)!r}",
           f"#define AGB_MUL1 {float(mul1)!r}",
           arr("AGB_PREFACT", pref),
           arr("AGB_COEF", coef),
           arr("AGB_NORM", norm),
           arr("AGB_SEED", seed),
           arr("AGB_SEED_F", seed, "float"),
           arr("AGB_ALPHA", alpha),
           arr("AGB_BETA", beta),
           arr("AGB_ALPHA_F", alpha, "float"),
           arr("AGB_BETA_F", beta, "float"),
           arr("AGB_NBETAQ", nbetaq),
           arr("AGB_NBETAQ_F", nbetaq, "float"),
           f"#define AGB_SKIP_N {LMAX // 2 + 1}",
           arr2("AGB_SKIP", skip),
           arr2("AGB_SKIP_F", skip, "float2", "f")]
    out_path.write_text("\n".join(src))


if __name__ == "__main__":
    main(Path(__file__).with_name("legendre_tables.cuh"))
