"""Writes logtab.h: the reduction table of the two-phase correctly rounded log in ddmath.cuh.

Run from this directory: ``python gen_logtab.py > logtab.h``.  Exact arithmetic only (Python's
``decimal`` at 80 digits and integer bit patterns), so the output is the same on every machine.

Reduction (Tang's table-driven method, P. T. P. Tang, "Table-driven implementation of the
logarithm function in IEEE floating-point arithmetic", ACM TOMS 16, 1990):
  x = 2^k z with z in [Z0, 2 Z0), Z0 = the double with bits kOff; the bit pattern u - kOff of x splits
  into k (its top 12 bits) and the subinterval index i (the next 8), so the 256 subintervals are
  contiguous ranges of bit patterns.
  For each subinterval, invc_i is a multiple of 2^-8 near 1/z, so r = z * invc_i - 1 is exact in one
  fma: z * invc_i - 1 is an integer multiple of 2^-61 (z < 1) or 2^-60 (z >= 1), and |r| < 2^-8
  (resp. 2^-7) keeps that integer below 2^53.  This script checks the bound at both ends of every
  subinterval (r is monotone in z).
  log x = k ln 2 + logc_i + log1p(r), logc_i = -log(invc_i) in two doubles (hi + lo, 2^-106).
  kOff is chosen so that z = 1 lies in the middle of its subinterval, whose invc is exactly 1: near
  x = 1, log x = log1p(x - 1) with no cancellation against a table value.
"""
from decimal import Decimal, getcontext
import struct

getcontext().prec = 80

N_BITS = 8
N = 1 << N_BITS
SHIFT = 52 - N_BITS
# 0x3FE6000000000000 (z0 = 0.6875) moved back by half a subinterval, so that 1.0 is a midpoint
K_OFF = 0x3FE6000000000000 - (1 << (SHIFT - 1))


def bits_to_double(u):
    return struct.unpack("<d", struct.pack("<Q", u))[0]


def hexd(x):
    return float.hex(x)


def dd(v):
    """v (Decimal) as hi + lo doubles, each correctly rounded."""
    hi = float(v)
    lo = float(v - Decimal(hi))
    return hi, lo


def main():
    u_one = 0x3FF0000000000000
    i_one = ((u_one - K_OFF) >> SHIFT) & (N - 1)
    assert ((u_one - K_OFF) & ((1 << SHIFT) - 1)) == 1 << (SHIFT - 1), "1.0 not at a subinterval midpoint"
    rows = []
    rmax = Decimal(0)
    for i in range(N):
        ulo = K_OFF + (i << SHIFT)
        uhi = ulo + (1 << SHIFT) - 1
        zlo, zhi = Decimal(bits_to_double(ulo)), Decimal(bits_to_double(uhi))
        if i == i_one:
            invc = Decimal(1)
        else:
            zmid = (zlo + zhi) / 2
            invc = Decimal(round((1 / zmid) * 256)) / 256
        for z in (zlo, zhi):
            r = z * invc - 1
            bound = Decimal(2) ** -8 if z < 1 else Decimal(2) ** -7
            assert abs(r) < bound, (i, z, r)
            rmax = max(rmax, abs(r))
        lh, ll = dd(-invc.ln()) if i != i_one else (0.0, 0.0)
        rows.append((float(invc), lh, ll))
    ln2 = Decimal(2).ln()
    # ln 2 with 42 significant bits (k ln2_hi is exact for |k| < 2^11), then the rest in two doubles
    ln2_hi = Decimal(int(ln2 * (1 << 42))) / (1 << 42)
    ln2_lo, ln2_lo2 = dd(ln2 - ln2_hi)
    ln2_dd = dd(ln2)
    third = dd(Decimal(1) / 3)
    print("// Generated by gen_logtab.py (exact decimal arithmetic); do not edit by hand.")
    print("// Reduction table of the two-phase correctly rounded log (ddmath.cuh): for the 256 subintervals")
    print("// of bit patterns u - kLogOff, {invc, -log(invc) hi, -log(invc) lo}.")
    print(f"// max |r| over all subintervals: {float(rmax):.6g} (2^{float(rmax.ln() / ln2):.3f})")
    print("#pragma once")
    print("namespace bgpu {")
    print("namespace dd {")
    print(f"constexpr unsigned long long kLogOff = 0x{K_OFF:016X}ull;")
    print(f"constexpr int kLogTabBits = {N_BITS};")
    print(f"constexpr int kLogTabN = {N};")
    print(f"constexpr double kLn2Hi42 = {hexd(float(ln2_hi))};  // 42 significant bits")
    print(f"constexpr double kLn2Lo = {hexd(ln2_lo)};")
    print(f"constexpr double kLn2Lo2 = {hexd(ln2_lo2)};")
    print(f"constexpr double kLn2DDHi = {hexd(ln2_dd[0])};")
    print(f"constexpr double kLn2DDLo = {hexd(ln2_dd[1])};")
    print(f"constexpr double kThirdHi = {hexd(third[0])};")
    print(f"constexpr double kThirdLo = {hexd(third[1])};")
    print("#define BGPU_LOGTAB_ROWS \\")
    for j, (a, b, c) in enumerate(rows):
        end = ", \\" if j + 1 < N else ""
        print(f"  {hexd(a)}, {hexd(b)}, {hexd(c)}{end}")
    print("}  // namespace dd")
    print("}  // namespace bgpu")


if __name__ == "__main__":
    main()
