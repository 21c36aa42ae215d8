"""The arithmetic behind the parallel PageRank that reproduces the
reference's sequential FP32 sums (k_pr_hub_exact in pagerank.cu), modelled
on the CPU and checked against a plain sequential fold.

The reference sums each vertex's messages one after another in float
(MPG/CPUFunctorHoster.cpp:21-26).  The messages are non-negative, so the
running sum s only grows.  While s stays in one binade [2^k, 2^(k+1)),
every representable value there is an integer multiple of u = ulp(s), and
fl(s + x) = s + u * round(x / u) unless x / u ends in exactly one half (a
tie, rounded to even by s's last bit).  So a run of additions that never
leaves the binade and meets no tie is s + u * (sum of integers): an integer
prefix sum, computable in parallel.  The first thread whose prefix reaches
2^24 units (the binade's end) or that holds a tie folds its own elements
with ordinary float adds from the exact running sum; the threads after it
then rescan in the new binade.  This file restates that procedure in
Python with the kernel's thread and chunk structure and checks, bit for
bit, that it equals the sequential fold on many inputs, ties and binade
crossings included."""
import numpy as np
import pytest


def q_units(x, ks):
    """round(x / u) for u = 2^(ks-150) (the ulp of a float with biased
    exponent ks), clamped to 2^23; and whether x / u ends in exactly .5."""
    bx = int(np.float32(x).view(np.uint32))
    ex = bx >> 23
    if ex == 0:
        m, ex = bx & 0x7FFFFF, 1
    else:
        m = (bx & 0x7FFFFF) | 0x800000
    d = ks - ex
    if d < 0:
        return 1 << 23, False
    if d == 0:
        return min(m, 1 << 23), False
    if d > 24:
        return 0, False
    r = m & ((1 << d) - 1)
    h = 1 << (d - 1)
    return min((m >> d) + (1 if r > h else 0), 1 << 23), r == h


def seq_fold(xs, s=np.float32(0)):
    s = np.float32(s)
    for x in xs:
        s = np.float32(s + np.float32(x))
    return s


def exact_fold(xs, T=8, K=4, head=16):
    """The kernel's procedure: a serial head, then chunks of T*K elements,
    thread t owning elements [t*K, t*K+K) of a chunk."""
    xs = np.asarray(xs, np.float32)
    n = len(xs)
    s = seq_fold(xs[:min(n, head)])
    pos = head
    rescans = 0
    while pos < n:
        chunk = np.zeros(T * K, np.float32)
        m = min(T * K, n - pos)
        chunk[:m] = xs[pos:pos + m]
        start = 0
        while start < T:
            rescans += 1
            bits = int(s.view(np.uint32))
            ks = bits >> 23
            base = (bits & 0x7FFFFF) | 0x800000
            L = np.zeros(T, np.int64)
            tie = np.zeros(T, bool)
            for t in range(start, T):
                tot = 0
                for k in range(K):
                    qq, tt = q_units(chunk[t * K + k], ks)
                    tot += qq
                    tie[t] |= tt
                L[t] = min(tot, 1 << 23)
            incl = np.cumsum(L)
            assert incl[-1] < 2 ** 32  # the kernel's uint32 scan cannot overflow
            bad = [t for t in range(start, T) if ks == 0 or tie[t] or base + incl[t] >= 1 << 24]
            if not bad:
                s = np.uint32((ks << 23) | ((base + int(incl[-1])) & 0x7FFFFF)).view(np.float32)
                break
            c = bad[0]
            prefix = int(incl[c] - L[c])
            s2 = s if c == start else np.uint32((ks << 23) | ((base + prefix) & 0x7FFFFF)).view(np.float32)
            s = seq_fold(chunk[c * K:(c + 1) * K], s2)
            start = c + 1
        pos += T * K
    return s, rescans


def _cases():
    rng = np.random.default_rng(12345)
    out = []
    for n in (1, 5, 16, 17, 40, 100, 257, 1000, 5000):
        out.append(rng.random(n, dtype=np.float32) * np.float32(1e-6))
    # PageRank-like: rank / outdeg
    for n in (300, 3000):
        rk = np.float32(0.15) + rng.random(n).astype(np.float32)
        od = rng.integers(1, 50, n).astype(np.float32)
        out.append((rk / od).astype(np.float32))
    # wide magnitudes, zeros, a huge term late (crossing several binades)
    x = (rng.random(2000) ** 8).astype(np.float32)
    x[::7] = 0
    x[1500] = np.float32(1e3)
    out.append(x)
    # identical terms (many ties once s outgrows them)
    out.append(np.full(3000, np.float32(1.0)))
    out.append(np.full(3000, np.float32(0.75)))
    # powers of two: exact ties at every scale
    out.append(np.float32(2.0) ** -rng.integers(0, 30, 2500).astype(np.float32))
    return out


@pytest.mark.parametrize("i", range(len(_cases())))
@pytest.mark.parametrize("T,K,head", [(8, 4, 16), (4, 2, 0), (32, 8, 64)])
def test_exact_fold_equals_sequential_fold(i, T, K, head):
    xs = _cases()[i]
    want = seq_fold(xs)
    got, _ = exact_fold(xs, T, K, head)
    assert got.view(np.uint32) == want.view(np.uint32), (got, want)


def test_ties_are_rounded_to_even():
    # s = 2^24 (ulp 2): adding 1.0 is an exact tie each time; the sequential
    # fold rounds to even, so s stays 2^24
    xs = np.concatenate([[np.float32(2.0 ** 24)], np.ones(64, np.float32)])
    want = seq_fold(xs)
    assert want == np.float32(2.0 ** 24)
    got, _ = exact_fold(xs, 4, 4, 1)
    assert got == want


def test_rescans_stay_logarithmic():
    """After the head, binade crossings (and so rescans) grow with log2(n),
    not n: a chunk costs one scan unless it crosses."""
    rng = np.random.default_rng(7)
    xs = (rng.random(60000, dtype=np.float32) + np.float32(0.5)) * np.float32(1e-7)
    got, rescans = exact_fold(xs, 64, 8, 512)
    assert got == seq_fold(xs)
    chunks = -(-(len(xs) - 512) // 512)
    assert rescans <= chunks + 3 * 8
