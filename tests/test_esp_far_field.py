"""The ESP kernels evaluate a primitive pair as a point multipole (asymptotic
Boys forms, no exponential) once T = p |P - C|^2 reaches far_T(L) for its
angular class L = l_a + l_b (chemtoolscuda_b200/csrc/ctc_esp.cu).  These tests
pin that threshold: at and beyond it, F_0 = sqrt(pi / T) / 2 and
F_n = (2n - 1) / (2T) F_{n-1} agree with the Boys function to 2e-17 relative
for every n <= L, computed here from the incomplete gamma function in 40-digit
arithmetic (F_n(T) = gamma(n + 1/2, T) / (2 T^(n + 1/2)), lower incomplete)."""
import os
import re

import pytest

mpmath = pytest.importorskip("mpmath")

SRC = os.path.join(os.path.dirname(__file__), "..", "chemtoolscuda_b200", "csrc", "ctc_esp.cu")


def far_threshold():
    """(a, b) of far_T(L) = a + b L, read from the kernel source."""
    src = open(SRC).read()
    m = re.search(r"constexpr double far_T\(int L\) \{ return ([0-9.]+) \+ ([0-9.]+) \* L; \}", src)
    assert m, "far_T(L) not found in ctc_esp.cu"
    return float(m.group(1)), float(m.group(2))


def boys_exact(n, T):
    T = mpmath.mpf(T)
    return mpmath.gammainc(n + mpmath.mpf(1) / 2, 0, T) / (2 * T ** (n + mpmath.mpf(1) / 2))


def boys_asymptotic(L, T):
    T = mpmath.mpf(T)
    F = [mpmath.sqrt(mpmath.pi / T) / 2]
    for n in range(1, L + 1):
        F.append((2 * n - 1) / (2 * T) * F[-1])
    return F


@pytest.mark.parametrize("L", range(9))
def test_far_field_boys_forms_hold_beyond_the_threshold(L):
    mpmath.mp.dps = 40
    a, b = far_threshold()
    T0 = a + b * L
    for T in (T0, T0 + 0.37, T0 + 3.0, 2 * T0, 1e3):
        Fa = boys_asymptotic(L, T)
        for n in range(L + 1):
            rel = abs(Fa[n] / boys_exact(n, T) - 1)
            assert rel <= 2e-17, (L, T, n, float(rel))


@pytest.mark.parametrize("L", [0, 4, 8])
def test_threshold_is_needed(L):
    """Well below the threshold the asymptotic forms are measurably wrong, so
    the near-field branch (Taylor table + downward recursion) is required."""
    mpmath.mp.dps = 40
    T = 35.0 - 3.0 * (L == 0)
    Fa = boys_asymptotic(L, T)
    worst = max(abs(Fa[n] / boys_exact(n, T) - 1) for n in range(L + 1))
    assert worst > 1e-16
