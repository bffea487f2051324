"""Generate ctc_ao_poly.inc: per-type AO polynomial evaluators with literal exponents.

For every segment type (s, p, Cartesian/pure d, f, g) one device function
evaluates all components and, depending on DERIV, their first and second
derivatives (written to o[q * ld_q + component * ldc]), given powers X[i] = x^(i-2) (X[0] = X[1] = 0), the same for y and
z, and the contracted radial sums R0, R1, R2 (see ctc_ao.cu).  With TRACK = 1
the running maximum of the high word of |value| (sign cleared; its exponent is
the exponent of the largest |value|) over the components is kept in mx[0], with
TRACK = 4 also those of the three first derivatives in mx[1..3] (the row
scales of the tensor-core split operands).  The terms come
from gen_terms.py; writing their exponents as literals lets the compiler keep
the power arrays in registers.

    python chemtoolscuda_b200/csrc/gen_ao_poly.py > chemtoolscuda_b200/csrc/ctc_ao_poly.inc
"""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from gen_terms import TYPES, comps  # noqa: E402


def emit_type(ti, l, pure):
    cs = comps(l, pure)
    out = [f"// type {ti}: l = {l}{' (pure)' if pure else ''}, {len(cs)} components",
           "template <int DERIV, int TRACK>",
           f"__device__ __forceinline__ void ao_poly_{ti}(const double* X, const double* Y, const double* Z,",
           "    double R0, double R1, double R2, double* __restrict__ o, int64_t ld_q, int64_t ldc, int nq_out,",
           "    unsigned* mx) {"]
    for j, comp in enumerate(cs):
        out.append("  {")
        out.append("    double q0 = 0.0, q1 = 0.0, q2 = 0.0, q3 = 0.0, q4 = 0.0, q5 = 0.0, q6 = 0.0, q7 = 0.0, q8 = 0.0, q9 = 0.0;")
        for (c, a, b, z) in comp:
            C = repr(float(c))
            out.append(f"    q0 += {C} * X[{a+2}] * Y[{b+2}] * Z[{z+2}] * R0;")
            out.append("    if (DERIV >= 1) {")
            out.append(f"      const double Xa = {a}.0 * X[{a+1}], Xb = X[{a+3}], Ya = {b}.0 * Y[{b+1}], Yb = Y[{b+3}], Za = {z}.0 * Z[{z+1}], Zb = Z[{z+3}];")
            out.append(f"      q1 += {C} * Y[{b+2}] * Z[{z+2}] * (Xa * R0 - 2.0 * Xb * R1);")
            out.append(f"      q2 += {C} * X[{a+2}] * Z[{z+2}] * (Ya * R0 - 2.0 * Yb * R1);")
            out.append(f"      q3 += {C} * X[{a+2}] * Y[{b+2}] * (Za * R0 - 2.0 * Zb * R1);")
            out.append("      if (DERIV >= 2) {")
            out.append(f"        q4 += {C} * Y[{b+2}] * Z[{z+2}] * ({a*(a-1)}.0 * X[{a}] * R0 - {2*(2*a+1)}.0 * X[{a+2}] * R1 + 4.0 * X[{a+4}] * R2);")
            out.append(f"        q5 += {C} * Z[{z+2}] * (Xa * Ya * R0 - 2.0 * (Xa * Yb + Xb * Ya) * R1 + 4.0 * Xb * Yb * R2);")
            out.append(f"        q6 += {C} * Y[{b+2}] * (Xa * Za * R0 - 2.0 * (Xa * Zb + Xb * Za) * R1 + 4.0 * Xb * Zb * R2);")
            out.append(f"        q7 += {C} * X[{a+2}] * Z[{z+2}] * ({b*(b-1)}.0 * Y[{b}] * R0 - {2*(2*b+1)}.0 * Y[{b+2}] * R1 + 4.0 * Y[{b+4}] * R2);")
            out.append(f"        q8 += {C} * X[{a+2}] * (Ya * Za * R0 - 2.0 * (Ya * Zb + Yb * Za) * R1 + 4.0 * Yb * Zb * R2);")
            out.append(f"        q9 += {C} * X[{a+2}] * Y[{b+2}] * ({z*(z-1)}.0 * Z[{z}] * R0 - {2*(2*z+1)}.0 * Z[{z+2}] * R1 + 4.0 * Z[{z+4}] * R2);")
            out.append("      }")
            out.append("    }")
        c = f"{j} * ldc"
        out.append(f"    o[{c}] = q0;")
        out.append(f"    if (DERIV >= 1) {{ if (nq_out > 1) {{ o[ld_q + {c}] = q1; o[2 * ld_q + {c}] = q2; o[3 * ld_q + {c}] = q3; }} }}")
        out.append(f"    if (DERIV >= 2) {{ if (nq_out > 4) {{ o[4 * ld_q + {c}] = q4; o[5 * ld_q + {c}] = q5; o[6 * ld_q + {c}] = q6;")
        out.append(f"      o[7 * ld_q + {c}] = q7; o[8 * ld_q + {c}] = q8; o[9 * ld_q + {c}] = q9; }} }}")
        out.append("    if (TRACK >= 1) mx[0] = max(mx[0], abs_hi(q0));")
        out.append("    if (TRACK >= 4 && DERIV >= 1) { mx[1] = max(mx[1], abs_hi(q1)); mx[2] = max(mx[2], abs_hi(q2)); mx[3] = max(mx[3], abs_hi(q3)); }")
        out.append("  }")
    out.append("}")
    return out


def main():
    print("// Generated by gen_ao_poly.py -- do not edit.")
    for ti, (l, pure) in enumerate(TYPES):
        print("\n".join(emit_type(ti, l, pure)))
        print()


if __name__ == "__main__":
    main()
