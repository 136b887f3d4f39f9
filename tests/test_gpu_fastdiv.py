"""The FP64 sweeps' arithmetic shortcuts give the same bits as plain IEEE arithmetic.

The sweeps take quotients that share a denominator (hv/h and hu/h; n^2/h^2 and hu*hv/h^2; the
three HLL components over one denominator) from one correctly rounded reciprocal with two
Markstein correction steps, and skip the limiter's division where the limiter saturates.  Parity
with the oracle needs every result bit-identical to IEEE division, so these tests run both forms
side by side on the GPU (include/paraclaws_b200.h: pcl_check_*):
  * > 10^8 pseudo-random quotient pairs over the method's whole range, the sweeps' range, zero and
    power-of-two numerators, all-ones-mantissa denominators and quotients near 1;
  * pairs constructed so that a/b lies within ~2^-40 ulp of a rounding midpoint (the hardest
    cases for a correction step), with random binade offsets;
  * the cell flux + HLL solve of both sweep directions, fast against plain, on random cells
    across the range the sweeps admit (including its ends and zero momenta), for the
    dam-break g and the ends of the g range the fast build accepts; the limiter with and without
    its saturation shortcut for all four limiter codes.
The tolerance is zero: any differing bit counts as a mismatch.
"""
import ctypes as C
import math

import numpy as np
import pytest

from paraclaws_b200 import _lib

pytestmark = pytest.mark.gpu


def near_midpoint_pairs(n: int, seed: int):
    """(a, b) with a/b = (2M+1)/2^53 * 2^k - t/(2^53 B) for an odd 53-bit B, a small odd t and a
    54-bit odd midpoint significand 2M+1: B*(2M+1) = A*2^53 + t exactly, so a = A*2^ea, b = B*2^eb
    puts a/b within |t|/B * 2^-53 ulp of the midpoint between two adjacent doubles."""
    rng = np.random.default_rng(seed)
    a = np.empty(n)
    b = np.empty(n)
    k = 0
    mod = 1 << 53
    while k < n:
        B = int(rng.integers(1 << 52, 1 << 53)) | 1
        t = int(rng.integers(-(1 << 12), 1 << 12)) | 1
        X = (t * pow(B, -1, mod)) % mod
        mid = X + mod                     # odd, in [2^53, 2^54)
        P = B * mid
        A = (P - t) >> 53                 # exact: P - t = 0 mod 2^53
        if not (1 << 52) <= A < (1 << 53):
            continue
        ea = int(rng.integers(-60, 60))
        eb = int(rng.integers(-60, 60))
        sa = -1.0 if rng.random() < 0.5 else 1.0
        sb = -1.0 if rng.random() < 0.5 else 1.0
        a[k] = sa * math.ldexp(float(A), ea - 52)
        b[k] = sb * math.ldexp(float(B), eb - 52)
        k += 1
    return a, b


def test_random_quotients_match_ieee_division():
    L = _lib.load()
    bad, used = C.c_longlong(), C.c_longlong()
    for seed in (1, 2):
        assert L.pcl_check_quotients_random(1 << 27, seed, C.byref(bad), C.byref(used)) == 0
        assert used.value > 0.9 * (1 << 27), used.value
        assert bad.value == 0, f"{bad.value} of {used.value} quotients differ from IEEE division (seed {seed})"


def test_near_midpoint_quotients_match_ieee_division():
    L = _lib.load()
    a, b = near_midpoint_pairs(200_000, seed=5)
    # the construction really lands next to midpoints: a/b is never an exact double here
    bad, used = C.c_longlong(), C.c_longlong()
    assert L.pcl_check_quotients(a.ctypes.data, b.ctypes.data, len(a), C.byref(bad), C.byref(used)) == 0
    assert used.value == len(a)
    assert bad.value == 0, f"{bad.value} near-midpoint quotients differ from IEEE division"


def test_edge_quotients_match_ieee_division():
    L = _lib.load()
    vals = [0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 3.0, 1.0 / 3.0, np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0),
            np.nextafter(2.0, 0.0), 2.0 ** -64, 2.0 ** 63, 2.0 ** -960, 2.0 ** 959, 1e-10, 9.8100004196166992]
    a = np.array([x for x in vals for _ in vals])
    b = np.array([y for _ in vals for y in vals])
    bad, used = C.c_longlong(), C.c_longlong()
    assert L.pcl_check_quotients(a.ctypes.data, b.ctypes.data, len(a), C.byref(bad), C.byref(used)) == 0
    assert used.value > 0
    assert bad.value == 0


@pytest.mark.parametrize("grav", [float(np.float32(9.81)), 2.0 ** -20, 2.0 ** 20])
def test_fast_flux_path_matches_plain_path(grav):
    L = _lib.load()
    bad, fast, lim = C.c_longlong(), C.c_longlong(), C.c_longlong()
    n = 1 << 24
    assert L.pcl_check_flux_paths(n, 11, grav, C.byref(bad), C.byref(fast), C.byref(lim)) == 0
    assert fast.value > n // 4, fast.value  # most pairs take the fast path
    assert bad.value == 0, f"{bad.value} of {n} cell pairs: fast flux/HLL differs from the IEEE path"
    assert lim.value == 0, f"{lim.value} of {n} limited waves differ with the saturation shortcut"
