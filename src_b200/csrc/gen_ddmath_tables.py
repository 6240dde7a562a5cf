"""Writes sc_ddmath_tables.h: double-double constants for the table-driven
log and atan of sc_ddmath.cuh, evaluated with mpmath at 200 bits.

    python src_b200/csrc/gen_ddmath_tables.py

Each constant v is stored as (hi, lo) with hi = fl(v) and lo = fl(v - hi).
"""
import os

import mpmath as mp

mp.mp.prec = 200


def dd(v):
    hi = float(v)
    lo = float(v - mp.mpf(hi))
    return hi, lo


def fmt(x):
    return float.hex(x)


def main():
    out = []
    out.append("// Generated by gen_ddmath_tables.py (mpmath, 200-bit); do not edit.")
    out.append("#pragma once")
    out.append("namespace sc {")
    out.append("namespace ddm {")
    # log(j / 64) for j = 45 .. 91 (mantissas in [sqrt(1/2), sqrt(2)) round to these)
    out.append("// log(j / 64), j = 45 .. 91: {hi, lo}")
    out.append("constexpr int kLogJ0 = 45, kLogJ1 = 91;")
    out.append("SC_DDM_TABLE double kLogTab[kLogJ1 - kLogJ0 + 1][2] = {")
    for j in range(45, 92):
        h, l = dd(mp.log(mp.mpf(j) / 64))
        out.append(f"    {{{fmt(h)}, {fmt(l)}}},  // j = {j}")
    out.append("};")
    out.append("// 64 / j rounded to double, j = 45 .. 91 (reciprocals of the log table's centres)")
    out.append("SC_DDM_TABLE double kLogRcp[kLogJ1 - kLogJ0 + 1] = {")
    for j in range(45, 92):
        out.append(f"    {fmt(float(mp.mpf(64) / j))},  // j = {j}")
    out.append("};")
    out.append("// atan(j / 64), j = 0 .. 64: {hi, lo}")
    out.append("SC_DDM_TABLE double kAtanTab[65][2] = {")
    for j in range(0, 65):
        h, l = dd(mp.atan(mp.mpf(j) / 64))
        out.append(f"    {{{fmt(h)}, {fmt(l)}}},  // j = {j}")
    out.append("};")
    # ln2 split so that k * hi is exact for |k| < 2^11: hi keeps 42 significant bits
    m, e = mp.frexp(mp.log(2))
    hi = mp.ldexp(mp.floor(mp.ldexp(m, 42)), e - 42)
    lo_h, lo_l = dd(mp.log(2) - hi)
    out.append(f"constexpr double kLn2Hi = {fmt(float(hi))};  // 42 bits: k * kLn2Hi is exact")
    out.append(f"constexpr double kLn2Lo = {fmt(lo_h)};")
    out.append(f"constexpr double kLn2Lo2 = {fmt(lo_l)};")
    for name, v in (("kPiHalf", mp.pi / 2), ("kThird", mp.mpf(1) / 3), ("kHalf", mp.mpf(1) / 2)):
        h, l = dd(v)
        out.append(f"constexpr double {name}Hi = {fmt(h)}, {name}Lo = {fmt(l)};")
    out.append("}  // namespace ddm")
    out.append("}  // namespace sc")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sc_ddmath_tables.h")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
