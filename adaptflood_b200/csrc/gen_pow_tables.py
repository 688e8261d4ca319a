"""Generates af_pow_tables.h: the tables and polynomial coefficients of the
table-driven double-precision pow used on the FP64 parity path.

The reference computes the friction term with the C library's
pow(hflow, 10/3) (src/kernels.cpp:83,133).  On glibc >= 2.28 that pow is the
design of Szabolcs Nagy (Arm Optimized Routines, "pow" in the
optimized-routines project, MIT OR Apache-2.0 WITH LLVM-exception): x = 2^k z
with z in [0x1.69555p-1, 0x1.69555p0), log(x) = k ln2 + log(c) + log1p(z/c - 1)
from a 128-entry table of c chosen near the centre of each subinterval with a
short 1/c (so z/c - 1 is exact), carried as hi + lo; then
exp(y log x) = 2^(k/128) exp(r) from a 128-entry table of 2^(j/128) split as
H (1 + T).  This script restates the published construction of both tables
with mpmath, and fits the two polynomials (log1p(r) - r + r^2/2 on |r| <= the
largest reduced argument the table gives, relative error; exp(r) - 1 - r on
|r| <= ln2/256, absolute error) by its own Remez exchange.

Run:  python gen_pow_tables.py > af_pow_tables.h
"""
from __future__ import annotations

import mpmath as mp

mp.mp.dps = 80
N = 128  # entries of each table


def dbl(x) -> float:
    """Nearest double to the mpmath value x."""
    return float(mp.mpf(x))


def hexf(x: float) -> str:
    return float.hex(x)


def bits(x: float) -> int:
    import struct
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def from_bits(u: int) -> float:
    import struct
    return struct.unpack("<d", struct.pack("<Q", u & (2 ** 64 - 1)))[0]


# ------------------------------------------------------------------ log table
OFF = 0x3FE6955500000000  # bit pattern of 0x1.69555p-1, start of the z interval


def log_table():
    """Subinterval i holds the z whose bits satisfy ((ix - OFF) >> 45) % N == i.
    1/c = round(N/centre)/N below 1 and round(2N/centre)/(2N) above, so
    z*(1/c) - 1 is exact; log(c) is carried as logc (rounded to a multiple of
    2^-43, so k*ln2hi + logc is exact) plus logctail."""
    out = []
    for i in range(N):
        lo_bits = OFF + (i << 45)
        hi_bits = OFF + ((i + 1) << 45)
        # The subinterval straddling 1.0 wraps the binade: z values are
        # asdouble(ix - (tmp & 0xfff << 52)), so take the bit patterns as they
        # map into [0x1.69555p-1, 0x1.69555p0).
        zlo = mp.mpf(from_bits(lo_bits))
        zhi = mp.mpf(from_bits(hi_bits))
        centre = (zlo + zhi) / 2
        if centre < 1:
            invc = mp.nint(N / centre) / N
        else:
            invc = mp.nint(2 * N / centre) / (2 * N)
        c = 1 / invc
        lc = mp.log(c)
        logc = mp.nint(lc * mp.mpf(2) ** 43) / mp.mpf(2) ** 43
        logctail = lc - logc
        out.append((dbl(invc), dbl(logc), dbl(logctail), zlo, zhi, invc))
    return out


def max_reduced_arg(tab):
    m = mp.mpf(0)
    for (_, _, _, zlo, zhi, invc) in tab:
        m = max(m, abs(zlo * invc - 1), abs(zhi * invc - 1))
    return m


# ------------------------------------------------------------------ exp table
def exp_table():
    """2^(j/N) = H_j (1 + T_j) with H_j the nearest double; stored as the bits
    of T_j and the bits of H_j minus j << 45 (the exponent of 2^(k/N) is added
    back from k)."""
    out = []
    for j in range(N):
        v = mp.mpf(2) ** (mp.mpf(j) / N)
        H = dbl(v)
        T = dbl((v - mp.mpf(H)) / mp.mpf(H))
        out.append((bits(T), (bits(H) - (j << 45)) & (2 ** 64 - 1)))
    return out


# ------------------------------------------------------------------ Remez
def remez(f, w, deg, a, b, iters=30):
    """Minimax polynomial q of degree `deg` minimising max |w(x) (q(x) - f(x))|
    on [a, b] (Remez exchange, mpmath precision)."""
    n = deg + 2
    # Chebyshev-like start points, none at the centre (the weights used here vanish at 0)
    xs = [(a + b) / 2 + (b - a) / 2 * mp.cos(mp.pi * (n - 1 - i + mp.mpf(1) / 5) / (n - mp.mpf(1) / 2))
          for i in range(n)]
    coef = None
    for _ in range(iters):
        A = mp.matrix(n, n)
        rhs = mp.matrix(n, 1)
        for i, x in enumerate(xs):
            for k in range(deg + 1):
                A[i, k] = x ** k
            A[i, deg + 1] = (-1) ** i / w(x)
            rhs[i] = f(x)
        sol = mp.lu_solve(A, rhs)
        coef = [sol[k] for k in range(deg + 1)]

        def err(x):
            return w(x) * (mp.polyval(coef[::-1], x) - f(x))

        # locate the extrema of the error between sign changes on a fine grid
        grid = [a + (b - a) * mp.mpf(k) / 4000 for k in range(4001)]
        vals = [err(x) for x in grid]
        ext = []
        for k in range(len(grid)):
            left = vals[k - 1] if k > 0 else None
            right = vals[k + 1] if k + 1 < len(grid) else None
            v = vals[k]
            if (left is None or abs(v) >= abs(left)) and (right is None or abs(v) >= abs(right)):
                ext.append(k)
        # refine each extremum and keep an alternating set of n points
        pts = []
        for k in ext:
            lo = grid[max(k - 1, 0)]
            hi = grid[min(k + 1, len(grid) - 1)]
            if k == 0 or k == len(grid) - 1:
                x = grid[k]
            else:
                try:
                    x = mp.findroot(lambda t: mp.diff(err, t), grid[k], solver="secant")
                    if not (lo <= x <= hi):
                        x = grid[k]
                except Exception:  # noqa: BLE001
                    x = grid[k]
            pts.append((x, err(x)))
        alt = []
        for x, e in pts:
            if alt and mp.sign(alt[-1][1]) == mp.sign(e):
                if abs(e) > abs(alt[-1][1]):
                    alt[-1] = (x, e)
            else:
                alt.append((x, e))
        while len(alt) > n:
            if abs(alt[0][1]) < abs(alt[-1][1]):
                alt.pop(0)
            else:
                alt.pop()
        if len(alt) < n:
            break
        xs = [x for x, _ in alt]
    emax = max(abs(w(x) * (mp.polyval(coef[::-1], x) - f(x)))
               for x in [a + (b - a) * mp.mpf(k) / 2000 for k in range(2001)])
    return coef, emax


def log_poly(a):
    """log1p(r) ~ r - r^2/2 + r^3 (c3 + c4 r + ... + c8 r^5), relative error."""
    def f(r):
        if r == 0:
            return mp.mpf(1) / 3
        return (mp.log1p(r) - r + r * r / 2) / r ** 3

    def w(r):
        if r == 0:
            return mp.mpf(0)
        return abs(r ** 3 / mp.log1p(r))

    coef, e = remez(f, w, 5, -a, a)
    return coef, e


def exp_poly(a):
    """exp(r) ~ 1 + r + r^2 (C2 + C3 r + C4 r^2 + C5 r^3), absolute error."""
    def f(r):
        if r == 0:
            return mp.mpf(1) / 2
        return (mp.exp(r) - 1 - r) / r ** 2

    def w(r):
        return r * r

    coef, e = remez(f, w, 3, -a, a)
    return coef, e


def main():
    ltab = log_table()
    amax = max_reduced_arg(ltab)
    ln2 = mp.log(2)
    ln2hi = mp.nint(ln2 * mp.mpf(2) ** 43) / mp.mpf(2) ** 43
    ln2lo = ln2 - ln2hi
    lc, le = log_poly(amax)
    # evaluation form: p = ar3*(A1 + r A2 + ar2 (A3 + r A4 + ar2 (A5 + r A6)))
    # with ar = -r/2, ar2 = -r^2/2, ar3 = -r^3/2 (scalings by powers of two are exact)
    scale = [-2, -2, 4, 4, -8, -8]
    A = [-0.5] + [dbl(lc[k]) * scale[k] for k in range(6)]
    ea = ln2 / 256
    ec, ee = exp_poly(ea)
    C = [dbl(x) for x in ec]
    # exp argument reduction: x = k ln2/N + r; ln2/N split so k*hi is exact
    invln2N = dbl(1 / ln2) * N
    ln2N = ln2 / N
    ln2hiN = mp.nint(ln2N * mp.mpf(2) ** 43) / mp.mpf(2) ** 43
    ln2loN = ln2N - ln2hiN
    etab = exp_table()

    o = []
    o.append("// Generated by gen_pow_tables.py -- do not edit.")
    o.append("// Tables and coefficients of the table-driven FP64 pow (see af_pow.cuh).")
    o.append(f"// log1p fit: |r| <= {mp.nstr(amax, 8)}, relative error {mp.nstr(le, 4)}")
    o.append(f"// expm1 fit: |r| <= ln2/256, absolute error {mp.nstr(ee, 4)}")
    o.append("#pragma once")
    o.append(f"#define AF_POW_OFF 0x{OFF:016x}ULL")
    o.append(f"#define AF_POW_LN2HI {hexf(dbl(ln2hi))}")
    o.append(f"#define AF_POW_LN2LO {hexf(dbl(ln2lo))}")
    for k, a in enumerate(A):
        o.append(f"#define AF_POW_A{k} {hexf(a)}")
    for k, c in enumerate(C):
        o.append(f"#define AF_POW_C{k + 2} {hexf(c)}")
    o.append(f"#define AF_POW_INVLN2N {hexf(invln2N)}")
    o.append(f"#define AF_POW_NEGLN2HIN {hexf(-dbl(ln2hiN))}")
    o.append(f"#define AF_POW_NEGLN2LON {hexf(-dbl(ln2loN))}")
    o.append(f"#define AF_POW_SHIFT {hexf(float(3 * 2 ** 51))}")
    o.append("// X(invc, logc, logctail) for the 128 subintervals of z")
    o.append("#define AF_POW_LOG_TABLE(X) \\")
    for (invc, logc, tail, *_r) in ltab:
        o.append(f"  X({hexf(invc)}, {hexf(logc)}, {hexf(tail)}) \\")
    o.append("")
    o.append("// X(bits of T_j, bits of H_j - (j << 45)) for 2^(j/128) = H_j (1 + T_j)")
    o.append("#define AF_POW_EXP_TABLE(X) \\")
    for (t, s) in etab:
        o.append(f"  X(0x{t:016x}ULL, 0x{s:016x}ULL) \\")
    o.append("")
    print("\n".join(o))


if __name__ == "__main__":
    main()
