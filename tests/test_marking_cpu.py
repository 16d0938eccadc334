"""Refinement marking: the threshold of refine_fixed_fraction uses the total
the reference computes with Eigen's error.sum() (src/em_fwd.cc:1192).

The reference is built for plain x86-64 (no -march flags in its CMakeLists),
where Eigen sums a dynamic vector with SSE2 packets of two doubles: two packet
accumulators over pairs of packets, then a leftover packet, the two lanes, and
an odd last element.  With a sequential total the threshold -- and the flag
set -- can differ in the last bit.  The test searches seeded inputs for a case
where the two orders give different flags and checks that the library (and the
oracle) follow the packet order.
"""

import numpy as np

import emfem_b200 as E
import oracle as O


def _packet_sum(x):
    n = x.size
    if n < 2:
        return float(x[0]) if n == 1 else 0.0
    n1, n2 = n // 2 * 2, n // 4 * 4
    a0, a1 = float(x[0]), float(x[1])
    if n1 > 2:
        b0, b1 = float(x[2]), float(x[3])
        for i in range(4, n2, 4):
            a0 += float(x[i])
            a1 += float(x[i + 1])
            b0 += float(x[i + 2])
            b1 += float(x[i + 3])
        a0 += b0
        a1 += b1
        if n1 > n2:
            a0 += float(x[n2])
            a1 += float(x[n2 + 1])
    r = a0 + a1
    for i in range(n1, n):
        r += float(x[i])
    return r


def _seq_sum(x):
    r = 0.0
    for v in x:
        r += float(v)
    return r


def _flags(err, fraction, total):
    s = np.sort(err)[::-1]
    acc, thr = 0.0, 0.0
    for v in s:
        if acc < fraction * total:
            acc += float(v)
        else:
            thr = float(v)
            break
    return (err > thr).astype(np.uint8)


def _discriminating_case():
    rng = np.random.default_rng(11)
    for _ in range(20000):
        n = int(rng.integers(5, 40))
        err = np.exp(rng.uniform(-3, 3, n)) * rng.choice([1.0, 1e-9, 1e7], n)
        tp, ts = _packet_sum(err), _seq_sum(err)
        if tp == ts:
            continue
        s = np.sort(err)[::-1]
        cums = np.cumsum(s)
        for i in range(n - 1):
            for frac in (cums[i] / tp, np.nextafter(cums[i] / tp, 0), np.nextafter(cums[i] / tp, 1)):
                fp, fs = _flags(err, frac, tp), _flags(err, frac, ts)
                if not np.array_equal(fp, fs):
                    return err, float(frac), fp, fs
    raise AssertionError("no discriminating case found")


def test_packet_sum_matches_small_cases():
    for n in range(0, 12):
        x = np.arange(1, n + 1, dtype=np.float64) * 0.1
        assert abs(_packet_sum(x) - x.sum()) <= 1e-12 * max(1.0, abs(x.sum()))


def test_refine_fixed_fraction_uses_the_packet_order_total():
    err, frac, fp, fs = _discriminating_case()
    assert not np.array_equal(fp, fs)
    fg = E.refine_fixed_fraction(err, frac)
    fo = O.refine_fixed_fraction(err, frac)
    assert np.array_equal(fg, fp)
    assert np.array_equal(fo, fp)


def test_refine_fixed_fraction_random_vectors_agree_with_oracle():
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 4, 5, 7, 8, 9, 1000, 4097):
        err = rng.exponential(size=n)
        for frac in (0.05, 0.1, 0.5):
            fp = _flags(err, frac, _packet_sum(err))
            assert np.array_equal(E.refine_fixed_fraction(err, frac), fp)
            assert np.array_equal(O.refine_fixed_fraction(err, frac), fp)
