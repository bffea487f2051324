"""Generate ctc_terms.inc: polynomial terms of every AO component.

Each AO component of a segment is written as sum_t c_t x^a y^b z^c times the
contracted radial part sum_k coef_k exp(-alpha_k r^2), where coef_k already
holds N_l(alpha_k) = (2 alpha/pi)^(3/4) (4 alpha)^(l/2).  The angular factor
c_t is
  * Cartesian: 1/sqrt((2a-1)!! (2b-1)!! (2c-1)!!)   (src/cuda_basis_utils.cu:7-82)
  * pure:      S_lm coefficient / sqrt((2l-1)!!)     (src/cuda_basis_utils.cu:84-224)
with the reference's component order (src/evaluate_density.cu:80,114,143,196,
235-236,314) and the real solid harmonics of Helgaker, Jorgensen & Olsen,
Table 6.3, expanded into monomials.

    python chemtoolscuda_b200/csrc/gen_terms.py > chemtoolscuda_b200/csrc/ctc_terms.inc
"""
from math import sqrt


def dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


CART = {
    0: [(0, 0, 0)],
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
    3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (1, 2, 0), (2, 1, 0), (2, 0, 1), (1, 0, 2), (0, 1, 2),
        (0, 2, 1), (1, 1, 1)],
    4: [(0, 0, 4), (0, 1, 3), (0, 2, 2), (0, 3, 1), (0, 4, 0), (1, 0, 3), (1, 1, 2), (1, 2, 1),
        (1, 3, 0), (2, 0, 2), (2, 1, 1), (2, 2, 0), (3, 0, 1), (3, 1, 0), (4, 0, 0)],
}
s3, s15, s1p5, s2p5, s5, s35, s17p5 = sqrt(3), sqrt(15), sqrt(1.5), sqrt(2.5), sqrt(5), sqrt(35), sqrt(17.5)
PURE = {
    2: [  # m = 0, 1, -1, 2, -2
        [(1.0, 0, 0, 2), (-0.5, 2, 0, 0), (-0.5, 0, 2, 0)],
        [(s3, 1, 0, 1)],
        [(s3, 0, 1, 1)],
        [(0.5 * s3, 2, 0, 0), (-0.5 * s3, 0, 2, 0)],
        [(s3, 1, 1, 0)]],
    3: [  # m = 0, 1, -1, 2, -2, 3, -3
        [(1.0, 0, 0, 3), (-1.5, 2, 0, 1), (-1.5, 0, 2, 1)],
        [(2 * s1p5, 1, 0, 2), (-0.5 * s1p5, 3, 0, 0), (-0.5 * s1p5, 1, 2, 0)],
        [(2 * s1p5, 0, 1, 2), (-0.5 * s1p5, 2, 1, 0), (-0.5 * s1p5, 0, 3, 0)],
        [(0.5 * s15, 2, 0, 1), (-0.5 * s15, 0, 2, 1)],
        [(s15, 1, 1, 1)],
        [(0.5 * s2p5, 3, 0, 0), (-1.5 * s2p5, 1, 2, 0)],
        [(1.5 * s2p5, 2, 1, 0), (-0.5 * s2p5, 0, 3, 0)]],
    4: [  # m = 0, 1, -1, 2, -2, 3, -3, 4, -4
        [(1.0, 0, 0, 4), (0.375, 4, 0, 0), (0.375, 0, 4, 0), (0.75, 2, 2, 0), (-3.0, 2, 0, 2),
         (-3.0, 0, 2, 2)],
        [(2 * s2p5, 1, 0, 3), (-1.5 * s2p5, 3, 0, 1), (-1.5 * s2p5, 1, 2, 1)],
        [(2 * s2p5, 0, 1, 3), (-1.5 * s2p5, 2, 1, 1), (-1.5 * s2p5, 0, 3, 1)],
        [(1.5 * s5, 2, 0, 2), (-1.5 * s5, 0, 2, 2), (-0.25 * s5, 4, 0, 0), (0.25 * s5, 0, 4, 0)],
        [(3 * s5, 1, 1, 2), (-0.5 * s5, 3, 1, 0), (-0.5 * s5, 1, 3, 0)],
        [(0.5 * s17p5, 3, 0, 1), (-1.5 * s17p5, 1, 2, 1)],
        [(1.5 * s17p5, 2, 1, 1), (-0.5 * s17p5, 0, 3, 1)],
        [(s35 / 8, 4, 0, 0), (-6 * s35 / 8, 2, 2, 0), (s35 / 8, 0, 4, 0)],
        [(0.5 * s35, 3, 1, 0), (-0.5 * s35, 1, 3, 0)]],
}
# type index: 0 s, 1 p, 2 d, 3 5d, 4 f, 5 7f, 6 g, 7 9g
TYPES = [(0, False), (1, False), (2, False), (2, True), (3, False), (3, True), (4, False), (4, True)]


def comps(l, pure):
    if not pure:
        return [[(1.0 / sqrt(dfact(2 * a - 1) * dfact(2 * b - 1) * dfact(2 * c - 1)), a, b, c)]
                for (a, b, c) in CART[l]]
    n = 1.0 / sqrt(dfact(2 * l - 1))
    return [[(t[0] * n, t[1], t[2], t[3]) for t in comp] for comp in PURE[l]]


def main():
    terms, offs = [], []
    for l, pure in TYPES:
        row = []
        for comp in comps(l, pure):
            row.append(len(terms))
            terms.extend(comp)
        row.append(len(terms))
        offs.append(row + [row[-1]] * (16 - len(row)))
    print("// Generated by gen_terms.py -- do not edit.")
    print("// Define CTC_TERMS_HOST before including to get host arrays h_terms/h_comp_off")
    print("// instead of the __constant__ device arrays c_terms/c_comp_off.")
    print(f"#define CTC_NTERMS {len(terms)}")
    print("#ifdef CTC_TERMS_HOST")
    print("static const ctc::Term h_terms[CTC_NTERMS] = {")
    print("#else")
    print("__constant__ ctc::Term c_terms[CTC_NTERMS] = {")
    print("#endif")
    for c, a, b, z in terms:
        print(f"  {{{c!r}, {a}, {b}, {z}, 0}},")
    print("};")
    print("// [type][j] .. [type][j+1] are the terms of component j")
    print("#ifdef CTC_TERMS_HOST")
    print("static const int16_t h_comp_off[8][16] = {")
    print("#else")
    print("__constant__ int16_t c_comp_off[8][16] = {")
    print("#endif")
    for row in offs:
        print("  {" + ", ".join(str(x) for x in row) + "},")
    print("};")


if __name__ == "__main__":
    main()
