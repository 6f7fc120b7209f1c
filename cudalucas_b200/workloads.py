"""Synthetic workloads of the batched and serving modes.  The inputs of an LL
test are its exponent and iteration count, so these generators are the whole
data set: deterministic, seeded, no files."""
import numpy as np

from . import engine


def next_prime(v):
    v = int(v) | 1
    while not _is_prime(v):
        v += 2
    return v


def _is_prime(v):
    if v < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if v % p == 0:
            return v == p
    d, s = v - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17):
        x = pow(a, d, v)
        if x in (1, v - 1):
            continue
        for _ in range(s - 1):
            x = x * x % v
            if x == v - 1:
                break
        else:
            return False
    return True


def batch_exponents(count=256, lo=1e6, hi=2e7, seed=7):
    """`count` distinct primes, log-uniform in [lo, hi] (numpy default_rng(seed)
    over log10, each rounded up to the next prime), with the FFT length the
    length policy picks for each."""
    rng = np.random.default_rng(seed)
    out, seen = [], set()
    while len(out) < count:
        p = next_prime(10 ** rng.uniform(np.log10(lo), np.log10(hi)))
        if p in seen:
            continue
        seen.add(p)
        out.append((p, engine.choose_fft_length(p)))
    return out


def serve_requests(count=64, rate=50.0, lo=1e5, hi=5e7, iters=(1000, 50000), seed=11):
    """Poisson arrivals at `rate`/s; exponent prime log-uniform in [lo, hi];
    iterations uniform in `iters`.  Returns (arrival_s, p, n, iterations)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(count):
        t += rng.exponential(1.0 / rate)
        p = next_prime(10 ** rng.uniform(np.log10(lo), np.log10(hi)))
        k = int(rng.integers(iters[0], iters[1] + 1))
        out.append((t, p, engine.choose_fft_length(p), k))
    return out
