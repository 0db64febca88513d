"""Write radix_constants.cuh: cos/sin(2 pi q / R) for the odd FFT radices.

Run: python multiplescatteringcalculations_b200/csrc/gen_radix_constants.py
The values are correctly rounded doubles computed with mpmath at 50 digits.
"""
from pathlib import Path

import mpmath

mpmath.mp.dps = 50
RADICES = (3, 5, 7, 11)
lines = [
    "// Generated by gen_radix_constants.py: cos/sin(2*pi*q/R), q = 0..R-1, for the odd",
    "// FFT radices. Correctly rounded from 50-digit values.",
    "#pragma once",
    "namespace msc {",
    "template <int R> struct RadixTrig;",
]
for R in RADICES:
    c = [mpmath.cos(2 * mpmath.pi * q / R) for q in range(R)]
    s = [mpmath.sin(2 * mpmath.pi * q / R) for q in range(R)]
    fmt = lambda v: repr(float(v))  # noqa: E731
    lines.append(f"template <> struct RadixTrig<{R}> {{")
    lines.append(f"  static __host__ __device__ constexpr double c(int q) {{ constexpr double t[{R}] = {{" +
                 ", ".join(fmt(v) for v in c) + "}; return t[q]; }")
    lines.append(f"  static __host__ __device__ constexpr double s(int q) {{ constexpr double t[{R}] = {{" +
                 ", ".join(fmt(v) for v in s) + "}; return t[q]; }")
    lines.append("};")
lines.append("}  // namespace msc")
Path(__file__).with_name("radix_constants.cuh").write_text("\n".join(lines) + "\n")
