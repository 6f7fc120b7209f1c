// Host-side helpers of libllb200 (no GPU): exact residue extraction, digit
// canonicalisation and packing, checkpoint checksums and the FFT-length
// policy.  They mirror the semantics of CUDALucas's host code (cited per
// function) so that results and checkpoint files interoperate.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "../../include/llb200.h"

namespace {

// Bits of word j: floor(q/n) + 1 iff e_j = (-j*b) mod n < b (b = q mod n);
// CUDALucas.cu:1194-1220 derives the same bitmap from the weights.
struct WordBits {
  uint32_t q, n, b, qn;
  WordBits(uint32_t q_, uint32_t n_) : q(q_), n(n_), b(q_ % n_), qn(q_ / n_) {}
  // iterate e_j incrementally
  std::vector<uint8_t> all() const {
    std::vector<uint8_t> out(n);
    long long e = 0;
    for (uint32_t j = 0; j < n; ++j) {
      out[j] = (uint8_t)(qn + (e < (long long)b ? 1 : 0));
      e -= b;
      if (e < 0) e += n;
    }
    return out;
  }
};

// Full carry normalisation modulo 2^q-1: digits end in [0, 2^bits_j) and the
// value in [0, 2^q-1) (the all-ones pattern, which is 0 mod 2^q-1, becomes 0).
void normalise(std::vector<long long> &d, const std::vector<uint8_t> &bits) {
  const size_t n = d.size();
  for (int pass = 0; pass < 64; ++pass) {
    long long carry = 0;
    for (size_t j = 0; j < n; ++j) {
      long long v = d[j] + carry;
      const int b = bits[j];
      d[j] = v & ((1ll << b) - 1);
      carry = v >> b;
    }
    if (carry == 0) break;
    d[0] += carry;  // 2^q == 1 mod 2^q-1
  }
  bool ones = true;
  for (size_t j = 0; j < n && ones; ++j) ones = d[j] == (1ll << bits[j]) - 1;
  if (ones)
    for (size_t j = 0; j < n; ++j) d[j] = 0;
}

}  // namespace

extern "C" {

// Res64 of x * 2^-offset mod 2^q-1 (find_residue, CUDALucas.cu:1491-1534):
// the 64 bits of the canonical value starting at bit `offset`, wrapping at q.
uint64_t ll_digits_res64(const int32_t *digits, uint32_t q, uint32_t n, uint32_t offset) {
  if (!digits || !n || q <= n) return 0;
  WordBits wb(q, n);
  std::vector<uint8_t> bits = wb.all();
  std::vector<long long> d(digits, digits + n);
  normalise(d, bits);
  // bit position of word starts
  uint64_t res = 0;
  // locate word containing bit `offset`
  uint32_t w = (uint32_t)(((unsigned long long)offset * n) / q);
  uint32_t sw = (uint32_t)(((unsigned long long)w * q + n - 1) / n);
  int shift = (int)(offset - sw);
  int got = 0;
  unsigned __int128 acc = 0;
  int accbits = 0;
  uint32_t j = w;
  // first word: drop `shift` low bits
  acc = (unsigned __int128)((unsigned long long)d[j] >> shift);
  accbits = bits[j] - shift;
  while (accbits < 64) {
    j = (j + 1 == n) ? 0 : j + 1;
    acc |= (unsigned __int128)(unsigned long long)d[j] << accbits;
    accbits += bits[j];
  }
  (void)got;
  res = (uint64_t)acc;
  return res;
}

// standardize_digits (CUDALucas.cu:1465-1489), made exact: canonical digits,
// returns 1 when the value is 0 mod 2^q-1.
int32_t ll_digits_standardize(int32_t *digits, uint32_t q, uint32_t n) {
  if (!digits || !n) return 0;
  WordBits wb(q, n);
  std::vector<uint8_t> bits = wb.all();
  std::vector<long long> d(digits, digits + n);
  normalise(d, bits);
  int zero = 1;
  for (uint32_t j = 0; j < n; ++j) {
    digits[j] = (int32_t)d[j];
    if (d[j]) zero = 0;
  }
  return zero;
}

// pack_bits (CUDALucas.cu:1594-1614): little-endian bit stream of the digits.
void ll_pack_bits(const int32_t *digits, uint32_t *packed, uint32_t q, uint32_t n) {
  WordBits wb(q, n);
  std::vector<uint8_t> bits = wb.all();
  const uint32_t words = (q + 31) / 32;
  unsigned long long acc = 0;
  int k = 0;
  uint32_t o = 0;
  for (uint32_t i = 0; i < n; ++i) {
    acc += (unsigned long long)(uint32_t)digits[i] << k;
    k += bits[i];
    while (k >= 32 && o < words) {
      packed[o++] = (uint32_t)acc;
      acc >>= 32;
      k -= 32;
    }
  }
  if (o < words) packed[o++] = (uint32_t)acc;
  while (o < words) packed[o++] = 0;
}

// unpack_bits (CUDALucas.cu:1285-1311): digits in [0, 2^bits_j).
void ll_unpack_bits(const uint32_t *packed, int32_t *digits, uint32_t q, uint32_t n) {
  WordBits wb(q, n);
  std::vector<uint8_t> bits = wb.all();
  const uint32_t words = (q + 31) / 32;
  unsigned long long acc = 0;
  int k = 0;
  uint32_t o = 0;
  for (uint32_t i = 0; i < n; ++i) {
    while (k < bits[i]) {
      unsigned long long w = o < words ? packed[o] : 0;
      ++o;
      acc |= w << k;
      k += 32;
    }
    digits[i] = (int32_t)(acc & ((1ull << bits[i]) - 1));
    acc >>= bits[i];
    k -= bits[i];
  }
}

// balance_digits (CUDALucas.cu:1313-1342): digits >= half the word range
// become negative with a carry of +1 into the next word; the final carry
// goes to word 0.
void ll_balance_digits(int32_t *digits, uint32_t q, uint32_t n) {
  WordBits wb(q, n);
  std::vector<uint8_t> bits = wb.all();
  int carry = 0;
  for (uint32_t j = 0; j < n; ++j) {
    const int32_t full = 1 << bits[j];
    digits[j] += carry;
    carry = 0;
    if (digits[j] >= full / 2) {
      digits[j] -= full;
      carry = 1;
    }
  }
  digits[0] += carry;
}

// checkpoint_checksum (CUDALucas.cu:1712-1733): MSB-first CRC over the bytes,
// polynomial 0x04C11DB7, zero initial value, no final xor.  The bytes are
// taken as signed chars shifted arithmetically, exactly as the reference does.
uint32_t ll_checkpoint_checksum(const void *bytes, size_t len) {
  const signed char *s = (const signed char *)bytes;
  uint32_t c = 0;
  for (size_t i = 0; i < len; ++i)
    for (int j = 7; j >= 0; --j) {
      const uint32_t bit = ((uint32_t)(s[i] >> j)) & 1u;
      c = ((c >> 31) == bit) ? (c << 1) : ((c << 1) ^ 0x04C11DB7u);
    }
  return c;
}

// ch_sum (CUDALucas.cu:1735-1743)
uint32_t ll_additive_checksum(const uint32_t *words, size_t count) {
  uint32_t s = 0;
  for (size_t i = 0; i < count; ++i) s += words[i];
  return s;
}

// Exponent bounds of choose_fft_length (CUDALucas.cu:1034-1050): power-law
// fits of the smallest and largest usable word counts for exponent q.
void ll_fft_bounds(uint32_t q, uint32_t *lb, uint32_t *ub) {
  const double ff1 = 0.999 * 1024.0 * 0.0000357822505975293;
  const double ff2 = 0.99 * 1024.0 * 0.0002670641830112380;
  const double e1 = 1.022179977969700;
  const double e2 = 0.929905288591965;
  if (lb) *lb = (uint32_t)ceil(ff1 * exp(e1 * log((double)q)));
  if (ub) *ub = (uint32_t)floor(ff2 * exp(e2 * log((double)q)));
}

// The built-in FFT-length table of init_ffts (CUDALucas.cu:955-971), in K.
static const uint32_t k_default_mult[] = {
    1, 2, 4, 8, 10, 14, 16, 18, 20, 32, 36, 42, 48, 50, 56, 60, 64, 70, 80, 84, 96, 112, 120, 126, 128,
    144, 160, 162, 168, 180, 192, 224, 256, 288, 320, 324, 336, 360, 384, 392, 400, 448, 512, 576, 640, 648,
    672, 720, 768, 784, 800, 864, 896, 900, 1024, 1152, 1176, 1280, 1296, 1344, 1440, 1568, 1600, 1728, 1792,
    2048, 2160, 2304, 2352, 2592, 2688, 2880, 3024, 3136, 3200, 3584, 3600, 4096, 4320, 4608, 4704, 5120,
    5184, 5600, 5760, 6048, 6144, 6272, 6400, 6480, 7168, 7200, 7776, 8064, 8192, 8640, 9216, 9408, 10240,
    10368, 10584, 10800, 11200, 11520, 12096, 12288, 12544, 12960, 13824, 14336, 14400, 16384, 17496, 18144,
    19208, 19600, 20000, 20250, 21952, 23328, 23814, 24300, 24500, 25088, 25600, 26244, 27000, 27216, 28000,
    28672, 31104, 31250, 32000, 32400, 32768, 33614, 34992, 36000, 36288, 38416, 39200, 39366, 40500, 41472,
    42336, 43200, 43904, 47628, 49000, 50000, 50176, 51200, 52488, 54432, 55296, 56000, 57344, 60750, 62500,
    64000, 64800, 65536};

// The active length table: the built-in table, or the built-in table merged
// with a measured list (ll_fft_table_merge), as init_ffts builds g_ffts from
// `<gpu> fft.txt` (CUDALucas.cu:975-1021).  Guarded for callers on several
// host threads.
static std::mutex g_table_mu;
static std::vector<uint32_t> g_table;  // empty: the built-in table

static std::vector<uint32_t> active_table() {
  std::lock_guard<std::mutex> lock(g_table_mu);
  if (!g_table.empty()) return g_table;
  std::vector<uint32_t> t;
  for (uint32_t m : k_default_mult) t.push_back(m * 1024u);
  return t;
}

int32_t ll_fft_table(uint32_t *lengths, int32_t max_count) {
  const std::vector<uint32_t> t = active_table();
  if (lengths)
    for (int32_t i = 0; i < (int32_t)t.size() && i < max_count; ++i) lengths[i] = t[(size_t)i];
  return (int32_t)t.size();
}

// init_ffts (CUDALucas.cu:947-1022): the built-in lengths below the smallest
// measured length, then the measured lengths (ascending, as the benchmark
// writes them), then the built-in lengths above the largest measured one.
// Inside the measured range only measured lengths remain, so a length the
// benchmark found slower than a longer one is never chosen.  count == 0
// restores the built-in table.
int32_t ll_fft_table_merge(const uint32_t *measured, int32_t count) {
  if (count < 0 || (count > 0 && !measured)) return -1;
  std::vector<uint32_t> m;
  for (int32_t i = 0; i < count; ++i)
    if (measured[i] && (m.empty() || measured[i] > m.back())) m.push_back(measured[i]);
  std::vector<uint32_t> t;
  if (!m.empty()) {
    for (uint32_t d : k_default_mult)
      if (d * 1024u < m.front()) t.push_back(d * 1024u);
    t.insert(t.end(), m.begin(), m.end());
    for (uint32_t d : k_default_mult)
      if (d * 1024u > m.back()) t.push_back(d * 1024u);
  }
  std::lock_guard<std::mutex> lock(g_table_mu);
  g_table = t;
  return (int32_t)(t.empty() ? sizeof(k_default_mult) / sizeof(k_default_mult[0]) : t.size());
}

// The pruning of -cufftbench (CUDALucas.cu:2500-2513): scanning from the
// longest length down, a length is kept when it is faster than every longer
// length; lengths that are powers of two (in K) are always kept.
int32_t ll_fft_prune(const uint32_t *lengths, const float *ms_per_iter, int32_t count, int32_t *keep) {
  if (count < 0 || (count > 0 && (!lengths || !ms_per_iter || !keep))) return -1;
  float best = 0.f;
  bool any = false;
  int32_t kept = 0;
  for (int32_t i = count - 1; i >= 0; --i) {
    const uint32_t k = lengths[i] / 1024u;
    const bool pow2 = k && (k & (k - 1)) == 0 && lengths[i] % 1024u == 0;
    keep[i] = 0;
    if (ms_per_iter[i] > 0.f && (!any || ms_per_iter[i] < best)) {
      best = ms_per_iter[i];
      any = true;
      keep[i] = 1;
    } else if (pow2 && ms_per_iter[i] > 0.f) {
      keep[i] = 1;
    }
    kept += keep[i];
  }
  return kept;
}

// Largest exponent whose lower length bound (ll_fft_bounds) is at most n:
// the `max exp` column of `<gpu> fft.txt`.
uint32_t ll_fft_max_exponent(uint32_t n) {
  const double ff1 = 0.999 * 1024.0 * 0.0000357822505975293;
  const double e1 = 1.022179977969700;
  double qmax = exp(log((double)n / ff1) / e1);
  uint32_t q = qmax >= 4294967295.0 ? 0xfffffffdu : (uint32_t)qmax;
  uint32_t lb = 0;
  while (q > 3) {
    ll_fft_bounds(q, &lb, nullptr);
    if (lb <= n) break;
    --q;
  }
  return q;
}

// choose_fft_length (CUDALucas.cu:1027-1068): the smallest table length >=
// max(lb, want) that the engine supports, clamped to the upper bound.  A
// `want` that is not in the table is used as is when it lies within the
// bounds (init_ffts inserts it, CUDALucas.cu:995).
uint32_t ll_choose_fft_length(uint32_t q, uint32_t want) {
  uint32_t lb = 0, ub = 0;
  ll_fft_bounds(q, &lb, &ub);
  if (want && want >= lb && want <= ub && ll_length_supported(want)) return want;
  const std::vector<uint32_t> t = active_table();
  const uint32_t lo = want > lb ? want : lb;
  for (uint32_t n : t) {
    if (n < lo) continue;
    if (n > ub) break;
    if (ll_length_supported(n) && q > n) return n;
  }
  return 0;
}

}  // extern "C"
