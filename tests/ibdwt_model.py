"""Vectorised numpy model of the engine's two-pass IBDWT squaring, in the
engine's own HBM layout.  It is the floating-point reference the CUDA passes
are compared against (intermediate arrays within FP64 tolerance), and it is
checked itself against exact big-integer Lucas-Lehmer arithmetic.

Layout (N = n/2 complex elements, N = W*H):
  element m = m1*H + m2 holds words 2m (real part) and 2m+1 (imaginary part);
  the array at rest is A[k1][m2] (k1 in [0,W), m2 in [0,H)), address k1*H+m2.

Iteration = tall pass (column FFT over m2, Hermitian pairing + square, inverse
column FFT) followed by wide pass (inverse row FFT over k1, unweight, round,
two-step carry, -2, reweight, forward row FFT).

The weights follow CUDALucas.cu:1154-1185 (a_j = 2^(((-j*b) mod n)/n)); the
word sizes follow CUDALucas.cu:1194-1220 (word j is big iff e_j < b); the
-2 position follows CUDALucas.cu:1882-1886 (bit (offset+1) mod q after the
offset doubles).
"""
import numpy as np


def word_exponents(q, n):
    b = q % n
    j = np.arange(n, dtype=np.int64)
    return (-(j * b)) % n  # e_j, weight a_j = 2^(e_j/n)


def word_bits(q, n):
    b = q % n
    return (q // n) + (word_exponents(q, n) < b).astype(np.int64)


class Model:
    def __init__(self, q, n, W):
        assert n % 2 == 0
        self.q, self.n = q, n
        self.N = n // 2
        assert self.N % W == 0
        self.W, self.H = W, self.N // W
        assert self.W % 2 == 0 and self.H % 2 == 0
        e = word_exponents(q, n)
        self.e = e
        self.a = np.exp2(e / n)
        self.bits = word_bits(q, n)
        self.offset = 0

    # ---- layout helpers -------------------------------------------------
    def words_to_z(self, X):
        """word-order real array (n) -> z[m1][m2] complex (W x H)."""
        z = X[0::2] + 1j * X[1::2]          # z[m], m = m1*H + m2
        return z.reshape(self.W, self.H)    # [m1][m2]

    def z_to_words(self, z):
        flat = z.reshape(-1)
        X = np.empty(self.n)
        X[0::2] = flat.real
        X[1::2] = flat.imag
        return X

    # ---- passes ----------------------------------------------------------
    def forward_rows(self, z):
        """z[m1][m2] -> A[k1][m2] = sum_m1 z[m1][m2] w_W^(m1 k1), w = e^(+2pi i/W)."""
        return np.fft.ifft(z, axis=0) * self.W   # ifft uses e^{+i}

    def inverse_rows(self, A):
        return np.fft.fft(A, axis=0)             # e^{-i}, unnormalised

    def tall(self, A):
        W, H, N = self.W, self.H, self.N
        k1 = np.arange(W)[:, None]
        m2 = np.arange(H)[None, :]
        tw = np.exp(2j * np.pi * (k1 * m2) / N)
        C = A * tw
        Z = np.fft.ifft(C, axis=1) * H           # Z[k1][k2] = Z_{k1 + W k2}
        flat = Z.T.reshape(-1)                   # index k = k1 + W*k2
        k = np.arange(N)
        Zm = flat[(-k) % N]
        E = (flat + np.conj(Zm)) / 2
        O = (flat - np.conj(Zm)) / 2j
        P = E * E + np.exp(2j * np.pi * k / N) * O * O
        Q = 2j * E * O
        Zp = (P + Q).reshape(H, W).T             # back to [k1][k2]
        Cp = np.fft.fft(Zp, axis=1)              # inverse column DFT (e^{-i})
        return Cp * np.conj(tw)

    # ---- carry --------------------------------------------------------------
    def carry(self, Y, sub_word, sub_bit):
        """Y: unweighted, unnormalised conv output (word order, float).
        Returns (digits int64, max roundoff error)."""
        t = Y / (self.N * self.a)
        v = np.rint(t)
        err = np.max(np.abs(t - v))
        v = v.astype(np.int64)
        v[sub_word] -= (1 << sub_bit)
        b = self.bits
        n = self.n
        v0, v1 = v[0::2], v[1::2]
        b0, b1 = b[0::2], b[1::2]
        low0 = v0 & ((1 << b0) - 1); h0 = v0 >> b0
        low1 = v1 & ((1 << b1) - 1); h1 = v1 >> b1
        t1 = low1 + h0
        k1c = (t1 + (1 << (b1 - 1))) >> b1
        d1p = t1 - (k1c << b1)
        C1 = np.roll(h1, 1)     # incoming to element m from element m-1 (cyclic)
        C2 = np.roll(k1c, 1)
        t0 = low0 + C1
        k0 = (t0 + (1 << (b0 - 1))) >> b0
        d0p = t0 - (k0 << b0)
        d = np.empty(n, dtype=np.int64)
        d[0::2] = d0p + C2
        d[1::2] = d1p + k0
        return d, err

    # ---- LL --------------------------------------------------------------
    def load(self, digits, offset):
        self.offset = offset
        X = digits.astype(float) * self.a
        self.A = self.forward_rows(self.words_to_z(X))

    def start(self, offset=0):
        q, n = self.q, self.n
        pos = (offset + 2) % q
        d = np.zeros(n, dtype=np.int64)
        w = (pos * n) // q
        s = -((-w * q) // n)
        d[w] = 1 << (pos - s)
        self.load(d, offset)

    def sub_position(self):
        q, n = self.q, self.n
        pos = (self.offset + 1) % q
        w = (pos * n) // q
        s = -((-w * q) // n)
        return w, pos - s

    def iterate(self):
        self.offset = (2 * self.offset) % self.q
        A2 = self.tall(self.A)
        u = self.inverse_rows(A2)
        Y = self.z_to_words(u)
        w, bit = self.sub_position()
        d, err = self.carry(Y, w, bit)
        X = d.astype(float) * self.a
        self.A = self.forward_rows(self.words_to_z(X))
        self.digits = d
        return err


def digits_value(d, q, n):
    """Exact value mod 2^q-1 of a digit vector."""
    bits = word_bits(q, n)
    s = np.concatenate([[0], np.cumsum(bits)[:-1]])
    M = (1 << q) - 1
    x = 0
    for j in range(n - 1, -1, -1):
        x = (x << int(bits[j])) + int(d[j])
    return x % M


def exact_ll(q, k, offset=0):
    M = (1 << q) - 1
    s = 4
    for _ in range(k):
        s = (s * s - 2) % M
    return s
