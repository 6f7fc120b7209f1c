// B200 Lucas-Lehmer engine: two fused FP64 passes per iteration.
//
// Replaces one call of CUDALucas's lucas_square (CUDALucas.cu:1869-1986):
// cuFFT Z2Z -> square -> cuFFT Z2Z -> rcb -> splice, five launches that each
// sweep the n-word array, become two kernels that each read and write it once.
//
// Data layout (N = n/2 complex elements, N = W * H):
//   element m = m1*H + m2 holds words 2m (real) and 2m+1 (imaginary);
//   the array at rest is A[k1][m2] (k1 < W, m2 < H) at address k1*H + m2,
//   i.e. every column of the 2-D decomposition is contiguous in HBM.
//
// tall pass (one CTA per column pair k1, W-k1): twiddle w_N^(k1*m2), H-point
//   FFT, real-signal pairing of bins k and N-k with pointwise squaring (the
//   work of `square`, CUDALucas.cu:255-314), inverse H-point FFT, conjugate
//   twiddle.
// wide pass (one CTA per G consecutive rows m2): inverse W-point FFT,
//   unweight, round, roundoff max, -2, carry, reweight (the work of rcb and
//   splice, CUDALucas.cu:322-534), forward W-point FFT.
//
// Carries.  Word i keeps bal(low_i + c1_{i-1}) + c2_{i-1}, where c1 is the
// high part of word i-1's rounded value and c2 the carry out of balancing
// word i-1: the two-step carry that rcb applies inside its 128-word rows
// (CUDALucas.cu:389-405).  Element m's outgoing pair (c1, c2) depends only on
// element m's own two words, so the carry from the last row of CTA g to the
// first row of CTA g+1 (and from the top word to word 0, the 2^q == 1 wrap of
// carry_out[(blk+1) mod grid], CUDALucas.cu:474-483) is published once and
// read once: a single bounded wait per CTA, no serial chain.  (The generic
// kernels below hand over the pair packed in an int64; the specialised ones
// in kernels_static.cuh hand over the sum c1 + c2 as one double, which adds
// c2 before instead of after balancing word 0 -- the same value.)
//
// Consecutive passes are chained with programmatic dependent launch when a
// pass runs in a few waves: the next kernel's CTAs load their constant tables
// while the previous pass drains, and wait (griddepcontrol.wait) before they
// touch the state.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/llb200.h"
#include "fft_device.cuh"
#include "twiddle_consts.cuh"

namespace llb {

constexpr int EPT = 16;  // max elements per thread in one FFT stage

struct DevState {
  unsigned long long ticket;  // wide-pass CTA ticket counter (monotonic)
  uint32_t offset;            // shift of the current state (doubled by tall pass)
  uint32_t err_bits;          // max roundoff error (float bits), reset by host
  uint32_t fault;             // bit 0: wait timeout, bit 1: carry overflow
  uint32_t bar_count;         // grid barrier of the fused kernel: arrivals
  uint32_t bar_gen;           //   and generation
  uint32_t pad_;
};

struct TallArgs {
  double2 *A;
  const double2 *stw;   // stage twiddles of the specialised column transform
  const double2 *twH;   // e^{2 pi i e/H}
  const double2 *thi;   // e^{2 pi i (e<<TS)/N}
  const double2 *tlo;   // e^{2 pi i e/N}, e < 2^TS
  DevState *st;
  FftPlan ph;
  int W, H, N, ts, tmask;
  uint32_t q;
  int pf;  // > 0: prefetch into L2 the column pair pf units ahead (state larger than L2)
};

// Ready flags per wide-pass CTA: the specialised kernels hand the carry over
// warp by warp (at most 32 warps per CTA); the generic ones use the first.
constexpr int kWarpFlags = 32;

struct WideArgs {
  double2 *A;
  const double2 *stw;   // stage twiddles of the specialised row transform
  int32_t *xint;
  long long *carry;     // packed carries, one row of W per CTA
  uint32_t *flags;      // ready flags: kWarpFlags per CTA (one per warp)
  const double2 *twW;
  const int32_t *rowE;  // ((-(2*m2+t)*b) mod n), 2H entries
  const double *rowW;   // 2^(rowE/n)
  const double *rowWi;  // 2^(-rowE/n) / N
  const int32_t *colF;  // ((-2*H*m1*b) mod n), W entries
  const double *colW;
  const double *colWi;
  DevState *st;
  FftPlan pw;
  int W, H, G, ngroups;
  int pf;  // > 0: prefetch into L2 the row group pf tickets ahead (state larger than L2)
  uint32_t q, n, b, qn;
  // specialised kernels: column m1 = t + r*TR has exponent colF[t] - colD[r]
  // (mod n), i.e. weight colW[t] * colS[r] (times 2 when it wraps)
  int colD[16];
  double colS[16], colSi[16];
  double colS2[16], colSi2[16];  // 2*colS, 0.5*colSi (wrapped exponents)
};

__device__ __forceinline__ double2 omegaN(const double2 *__restrict__ thi, const double2 *__restrict__ tlo,
                                          int ts, int tmask, int e) {
  return cmul(__ldg(&thi[e >> ts]), __ldg(&tlo[e & tmask]));
}

// Real-signal pairing and squaring of bins k and N-k (w = w_N^k):
// E = (Z_k + conj Z_{N-k})/2, O = (Z_k - conj Z_{N-k})/(2i),
// Z'_k = E^2 + w O^2 + 2iEO, Z'_{N-k} = conj(E^2 + w O^2 - 2iEO).
__device__ __forceinline__ void pair_square(double2 &za, double2 &zb, double2 w) {
  double2 E = make_double2(0.5 * (za.x + zb.x), 0.5 * (za.y - zb.y));
  double2 O = make_double2(0.5 * (za.y + zb.y), -0.5 * (za.x - zb.x));
  double2 E2 = make_double2((E.x - E.y) * (E.x + E.y), 2.0 * E.x * E.y);
  double2 O2 = make_double2((O.x - O.y) * (O.x + O.y), 2.0 * O.x * O.y);
  double2 P = cadd(E2, cmul(w, O2));
  double2 EO = cmul(E, O);
  double2 Q = make_double2(-2.0 * EO.y, 2.0 * EO.x);
  za = cadd(P, Q);
  zb = conjg(csub(P, Q));
}

template <int EPT_>
__global__ void __launch_bounds__(256) tall_kernel(TallArgs a) {
  extern __shared__ double2 sm[];
  const int c = blockIdx.x;
  const int W = a.W, H = a.H;
  const bool special = (c == 0);
  const int kA = special ? 0 : c;
  const int kB = special ? W / 2 : W - c;
  if (c == 0 && threadIdx.x == 0) {
    // CUDALucas.cu:1882: offset <- 2*offset mod q, once per iteration
    const uint32_t o = a.st->offset;
    a.st->offset = (uint32_t)((2ull * o) % a.q);
  }
  for (int idx = threadIdx.x; idx < 2 * H; idx += blockDim.x) {
    const int col = idx >= H;
    const int m2 = idx - col * H;
    const int k1 = col ? kB : kA;
    double2 x = a.A[(size_t)k1 * H + m2];
    double2 w = omegaN(a.thi, a.tlo, a.ts, a.tmask, k1 * m2);
    sm[pad(idx)] = cmul(x, w);
  }
  __syncthreads();
  if (2 * H <= EPT_ * (int)blockDim.x) {
    fft_rows_b<EPT_, +1>(sm, a.ph, 2, 0, a.twH);
  } else {
    fft_rows_b<EPT_, +1>(sm, a.ph, 1, 0, a.twH);
    fft_rows_b<EPT_, +1>(sm, a.ph, 1, 1, a.twH);
  }
  if (!special) {
    for (int k2 = threadIdx.x; k2 < H; k2 += blockDim.x) {
      double2 za = sm[pad(k2)], zb = sm[pad(2 * H - 1 - k2)];
      pair_square(za, zb, omegaN(a.thi, a.tlo, a.ts, a.tmask, kA + W * k2));
      sm[pad(k2)] = za;
      sm[pad(2 * H - 1 - k2)] = zb;
    }
  } else {
    const int half = H / 2;
    for (int i = threadIdx.x; i <= half; i += blockDim.x) {  // column 0: k2 <-> (H-k2) mod H
      const int p = (H - i) % H;
      double2 za = sm[pad(i)], zb = sm[pad(p)];
      pair_square(za, zb, omegaN(a.thi, a.tlo, a.ts, a.tmask, W * i));
      sm[pad(i)] = za;
      if (p != i) sm[pad(p)] = zb;
    }
    for (int i = threadIdx.x; i < half; i += blockDim.x) {  // column W/2: k2 <-> H-1-k2
      double2 za = sm[pad(H + i)], zb = sm[pad(2 * H - 1 - i)];
      pair_square(za, zb, omegaN(a.thi, a.tlo, a.ts, a.tmask, W / 2 + W * i));
      sm[pad(H + i)] = za;
      sm[pad(2 * H - 1 - i)] = zb;
    }
  }
  __syncthreads();
  if (2 * H <= EPT_ * (int)blockDim.x) {
    fft_rows_b<EPT_, -1>(sm, a.ph, 2, 0, a.twH);
  } else {
    fft_rows_b<EPT_, -1>(sm, a.ph, 1, 0, a.twH);
    fft_rows_b<EPT_, -1>(sm, a.ph, 1, 1, a.twH);
  }
  for (int idx = threadIdx.x; idx < 2 * H; idx += blockDim.x) {
    const int col = idx >= H;
    const int m2 = idx - col * H;
    const int k1 = col ? kB : kA;
    double2 w = omegaN(a.thi, a.tlo, a.ts, a.tmask, k1 * m2);
    a.A[(size_t)k1 * H + m2] = cmulc(sm[pad(idx)], w);
  }
}

struct WordInfo {
  double w, wi;
  int bits;
};

__device__ __forceinline__ WordInfo word_info(const WideArgs &a, int jr, int f, double cw, double cwi) {
  WordInfo r;
  const int e = __ldg(&a.rowE[jr]) + f;
  const bool wrap = e >= (int)a.n;
  const int ee = wrap ? e - (int)a.n : e;
  r.w = __ldg(&a.rowW[jr]) * cw * (wrap ? 0.5 : 1.0);
  r.wi = __ldg(&a.rowWi[jr]) * cwi * (wrap ? 2.0 : 1.0);
  r.bits = (int)a.qn + (ee < (int)a.b ? 1 : 0);
  return r;
}

// Outgoing carry of an element: (c1, c2) packed as c1 * 2^24 + c2.
__device__ __forceinline__ long long pack_carry(long long c1, long long c2) { return (c1 << 24) + c2; }
__device__ __forceinline__ void unpack_carry(long long p, long long &c1, long long &c2) {
  c2 = (p << 40) >> 40;
  c1 = (p - c2) >> 24;
}

__device__ __forceinline__ long long element_carry(long long v0, long long v1, int b0, int b1, uint32_t &fault) {
  const long long h0 = v0 >> b0;
  const long long low1 = v1 & ((1ll << b1) - 1);
  const long long h1 = v1 >> b1;
  const long long t1 = low1 + h0;
  const long long k1 = (t1 + (1ll << (b1 - 1))) >> b1;
  if (k1 >= (1ll << 23) || k1 < -(1ll << 23) || h1 >= (1ll << 38) || h1 < -(1ll << 38)) fault |= 2u;
  return pack_carry(h1, k1);
}

__device__ __forceinline__ bool wait_flag(uint32_t *flag) {
  for (int it = 0; it < (1 << 24); ++it) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
    if (v) return true;
    __nanosleep(it < 64 ? 32 : 256);
  }
  return false;
}

enum { WIDE_ITER = 0, WIDE_REPORT = 1, WIDE_INIT = 2 };

template <int EPT_, int MODE>
__global__ void __launch_bounds__(256) wide_kernel(WideArgs a) {
  extern __shared__ double2 sm[];
  __shared__ int s_g;
  __shared__ float s_err[32];
  __shared__ uint32_t s_fault;
  if (threadIdx.x == 0) {
    s_fault = 0;
    s_g = MODE == WIDE_INIT ? (int)blockIdx.x : (int)(atomicAdd(&a.st->ticket, 1ull) % (unsigned long long)a.ngroups);
  }
  __syncthreads();
  const int g = s_g;
  const int W = a.W, H = a.H, G = a.G;
  const int m2b = g * G;
  longlong2 *smi = reinterpret_cast<longlong2 *>(sm);
  float emax = 0.f;
  uint32_t fault = 0;

  if (MODE != WIDE_INIT) {
    for (int idx = threadIdx.x; idx < G * W; idx += blockDim.x) {
      const int k1 = idx / G, r = idx - k1 * G;
      sm[pad(r * W + k1)] = a.A[(size_t)k1 * H + m2b + r];
    }
    __syncthreads();
    fft_rows_b<EPT_, -1>(sm, a.pw, G, 0, a.twW);

    // -2 at bit (offset+1) mod q (CUDALucas.cu:1882-1886), exact integer math
    const uint32_t off = a.st->offset;
    const uint32_t pos = (off + 1) % a.q;
    const uint32_t dw = (uint32_t)(((unsigned long long)pos * a.n) / a.q);
    const uint32_t sdw = (uint32_t)(((unsigned long long)dw * a.q + a.n - 1) / a.n);
    const long long sub = 1ll << (pos - sdw);

    // phase A: unweight, round, error, -2; keep rounded words in place
    for (int m1 = threadIdx.x; m1 < W; m1 += blockDim.x) {
      const int f = __ldg(&a.colF[m1]);
      const double cw = __ldg(&a.colW[m1]), cwi = __ldg(&a.colWi[m1]);
      for (int r = 0; r < G; ++r) {
        const int m2 = m2b + r;
        const WordInfo w0 = word_info(a, 2 * m2, f, cw, cwi);
        const WordInfo w1 = word_info(a, 2 * m2 + 1, f, cw, cwi);
        const double2 u = sm[pad(r * W + m1)];
        const double t0 = u.x * w0.wi, t1 = u.y * w1.wi;
        const double r0 = rint(t0), r1 = rint(t1);
        emax = fmaxf(emax, fabsf((float)(t0 - r0)));
        emax = fmaxf(emax, fabsf((float)(t1 - r1)));
        // no fraction bits left for the roundoff reading at 2^51 and above (or NaN)
        if (!(fabs(t0) < 0x1p51 && fabs(t1) < 0x1p51)) fault |= 2u;
        long long v0 = (long long)r0, v1 = (long long)r1;
        const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
        if (j0 == dw) v0 -= sub;
        if (j0 + 1 == dw) v1 -= sub;
        smi[pad(r * W + m1)] = make_longlong2(v0, v1);
        if (r == G - 1) a.carry[(size_t)g * W + m1] = element_carry(v0, v1, w0.bits, w1.bits, fault);
      }
    }
    __threadfence();
    __syncthreads();
    const int pred = g == 0 ? a.ngroups - 1 : g - 1;
    if (threadIdx.x == 0) {
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&a.flags[g]), "r"(1u) : "memory");
      if (!wait_flag(&a.flags[pred])) s_fault |= 1u;
      a.flags[pred] = 0;
    }
    __syncthreads();

    // phase B: carry in, balance, reweight (rows of this CTA in order)
    for (int m1 = threadIdx.x; m1 < W; m1 += blockDim.x) {
      const int f = __ldg(&a.colF[m1]);
      const double cw = __ldg(&a.colW[m1]), cwi = __ldg(&a.colWi[m1]);
      const int pm1 = g == 0 ? (m1 == 0 ? W - 1 : m1 - 1) : m1;
      long long cin = __ldcg(&a.carry[(size_t)pred * W + pm1]);
      for (int r = 0; r < G; ++r) {
        const int m2 = m2b + r;
        const WordInfo w0 = word_info(a, 2 * m2, f, cw, cwi);
        const WordInfo w1 = word_info(a, 2 * m2 + 1, f, cw, cwi);
        const longlong2 v = smi[pad(r * W + m1)];
        long long C1, C2;
        unpack_carry(cin, C1, C2);
        const int b0 = w0.bits, b1 = w1.bits;
        const long long low0 = v.x & ((1ll << b0) - 1), h0 = v.x >> b0;
        const long long low1 = v.y & ((1ll << b1) - 1);
        const long long t1 = low1 + h0;
        const long long k1c = (t1 + (1ll << (b1 - 1))) >> b1;
        const long long d1p = t1 - (k1c << b1);
        const long long t0 = low0 + C1;
        const long long k0 = (t0 + (1ll << (b0 - 1))) >> b0;
        const long long d0p = t0 - (k0 << b0);
        const long long d0 = d0p + C2, d1 = d1p + k0;
        cin = element_carry(v.x, v.y, b0, b1, fault);
        if (MODE == WIDE_REPORT) {
          const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
          a.xint[j0] = (int32_t)d0;
          a.xint[j0 + 1] = (int32_t)d1;
        }
        sm[pad(r * W + m1)] = make_double2((double)d0 * w0.w, (double)d1 * w1.w);
      }
    }
  } else {
    // start / resume: weighted digits (apply_weights, CUDALucas.cu:216-249)
    for (int m1 = threadIdx.x; m1 < W; m1 += blockDim.x) {
      const int f = __ldg(&a.colF[m1]);
      const double cw = __ldg(&a.colW[m1]), cwi = __ldg(&a.colWi[m1]);
      for (int r = 0; r < G; ++r) {
        const int m2 = m2b + r;
        const WordInfo w0 = word_info(a, 2 * m2, f, cw, cwi);
        const WordInfo w1 = word_info(a, 2 * m2 + 1, f, cw, cwi);
        const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
        sm[pad(r * W + m1)] = make_double2((double)a.xint[j0] * w0.w, (double)a.xint[j0 + 1] * w1.w);
      }
    }
  }
  __syncthreads();
  fft_rows_b<EPT_, +1>(sm, a.pw, G, 0, a.twW);
  for (int idx = threadIdx.x; idx < G * W; idx += blockDim.x) {
    const int k1 = idx / G, r = idx - k1 * G;
    a.A[(size_t)k1 * H + m2b + r] = sm[pad(r * W + k1)];
  }
  if (MODE != WIDE_INIT) {
    // block max of the roundoff error -> atomicMax on the float bits
#pragma unroll
    for (int o = 16; o; o >>= 1) emax = fmaxf(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    if ((threadIdx.x & 31) == 0) s_err[threadIdx.x >> 5] = emax;
    if (fault) atomicOr(&s_fault, fault);
    __syncthreads();
    if (threadIdx.x == 0) {
      float m = 0.f;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) m = fmaxf(m, s_err[i]);
      atomicMax(&a.st->err_bits, __float_as_uint(m));
      if (s_fault) atomicOr(&a.st->fault, s_fault);
    }
  }
}

#include "kernels_static.cuh"
#include "kernels_cluster.cuh"

// Registry of compile-time specialised kernels, by row length.
struct StaticWide {
  int L, G;
  void (*iter)(WideArgs);
  void (*report)(WideArgs);
  void (*init)(WideArgs);
  void (*iter_batch)(const WideArgs *, int);  // all members of a length class
  int nrad, rad[4];
  int extra;  // shared-memory entries beyond the rows (stage twiddles)
  int rows;   // shared-memory entries of the G rows
  int tr;     // threads per row (a thread's elements are t + r*tr)
  int alt;    // 1: the alternative row kernel of its length (LL_KERNELS_ALT_WIDE)
};
struct StaticTall {
  int L;
  void (*run)(TallArgs);
  void (*batch)(const TallArgs *, int);  // all members of a length class
  int nrad, rad[4];
  int tw;       // stage twiddle entries
  int smem;     // shared-memory entries of a CTA
  int threads;  // threads per CTA
  int ppc;      // column pairs per CTA
};

#define LLB_WIDE(LIST, G)                                                                                       \
  {LIST::L, G, wide_static<LIST, G, WIDE_ITER>, wide_static<LIST, G, WIDE_REPORT>, wide_static<LIST, G, WIDE_INIT>, \
   wide_static_batch<LIST, G>,                                                                                  \
   LIST::N, {LIST::a[0], LIST::a[1], LIST::N > 2 ? LIST::a[2 % LIST::N] : 0, 0}, tw_size<LIST>(),             \
   G * row_slots<LIST::L, G>(), LIST::L / 16, 0}
// rows through shared memory with few elements per thread (wide_any); MINB
// CTAs per SM asked of the register allocator
#define LLB_WIDE_ANY(LIST, G, MINB)                                                                         \
  {LIST::L, G, wide_any<LIST, G, MINB, WIDE_ITER>, wide_any<LIST, G, MINB, WIDE_REPORT>,                     \
   wide_any<LIST, G, MINB, WIDE_INIT>, wide_any_batch<LIST, G, MINB>,                                        \
   LIST::N, {LIST::a[0], LIST::N > 1 ? LIST::a[1 % LIST::N] : 0, LIST::N > 2 ? LIST::a[2 % LIST::N] : 0,       \
             LIST::N > 3 ? LIST::a[3 % LIST::N] : 0},                                                          \
   tw_size<LIST>(), G * row_slots<LIST::L, G>(), LIST::L / LIST::a[0], 1}
#define LLB_RAD(LIST)                                                                                 \
  LIST::N, {LIST::a[0], LIST::N > 1 ? LIST::a[1 % LIST::N] : 0, LIST::N > 2 ? LIST::a[2 % LIST::N] : 0, \
            LIST::N > 3 ? LIST::a[3 % LIST::N] : 0}
#define LLB_TALL(LIST) \
  {LIST::L, tall_static<LIST>, tall_static_batch<LIST>, LLB_RAD(LIST), tw_size<LIST>(),                      \
   padded(2 * LIST::L) + tall_extra<LIST>(), 2 * (LIST::L / 16), 1}
// the same without the batched variant (lengths that batches leave to
// solo launches: members without one run on their own branch)
#define LLB_TALL_ANY_SOLO(LIST, TC, PP)                                                                  \
  {LIST::L, tall_any<LIST, TC, PP>, nullptr, LLB_RAD(LIST), tw_size<LIST>(),                               \
   tall_any_smem<LIST, PP>(), 2 * PP * TC, PP}
// any radix list: TC threads per column, PP column pairs per CTA
#define LLB_TALL_ANY(LIST, TC, PP)                                                                       \
  {LIST::L, tall_any<LIST, TC, PP>, tall_any_batch<LIST, TC, PP>, LLB_RAD(LIST), tw_size<LIST>(),          \
   tall_any_smem<LIST, PP>(), 2 * PP * TC, PP}

using L256 = RList<16, 16>;
using L512 = RList<16, 2, 16>;
using L768 = RList<16, 3, 16>;
using L1024 = RList<16, 4, 16>;
using L1280 = RList<16, 5, 16>;
using L1536 = RList<16, 6, 16>;
using L1792 = RList<16, 7, 16>;
using L2048 = RList<16, 8, 16>;
using L2304 = RList<16, 9, 16>;
using L2560 = RList<16, 10, 16>;
using L3072 = RList<16, 12, 16>;
using L3584 = RList<16, 14, 16>;
using L4096 = RList<16, 16, 16>;
// column lengths of the tall_any kernels
using C24 = RList<4, 6>;
using C28 = RList<4, 7>;
using C100 = RList<10, 10>;
using C112 = RList<16, 7>;
using C120 = RList<12, 10>;
using C128 = RList<16, 8>;
using C140 = RList<14, 10>;
using C160 = RList<16, 10>;
using C168 = RList<14, 12>;
using C192 = RList<16, 12>;
using C224 = RList<16, 14>;
using C240 = RList<12, 10, 2>;
using C252 = RList<14, 9, 2>;
using C288 = RList<16, 9, 2>;
using C320 = RList<16, 10, 2>;
using C324 = RList<4, 9, 9>;
using C336 = RList<14, 12, 2>;
using C360 = RList<10, 9, 4>;
using C392 = RList<14, 14, 2>;
using C400 = RList<10, 10, 4>;
using C448 = RList<16, 14, 2>;
using C576 = RList<12, 12, 4>;
using C600 = RList<12, 10, 5>;
using C648 = RList<12, 9, 6>;
using C672 = RList<14, 12, 4>;
using C720 = RList<12, 10, 6>;
using C784 = RList<16, 7, 7>;
using C800 = RList<16, 10, 5>;
using C1568 = RList<16, 14, 7>;
using C2744 = RList<14, 14, 14>;
// columns of the long lengths (6048K and up): four stages at most, up to 486
// threads per column
using C1620 = RList<3, 9, 10, 6>;
using C1728 = RList<12, 12, 12>;
using C1800 = RList<5, 5, 12, 6>;
using C1944 = RList<3, 9, 12, 6>;
using C2160 = RList<5, 12, 6, 6>;
using C2240 = RList<14, 16, 10>;
using C2352 = RList<14, 14, 12>;
using C2400 = RList<5, 5, 16, 6>;
using C2592 = RList<3, 12, 12, 6>;
using C2688 = RList<14, 16, 12>;
using C2800 = RList<5, 5, 14, 8>;
using C2880 = RList<5, 12, 12, 4>;
using C2916 = RList<9, 9, 6, 6>;
using C3024 = RList<3, 14, 12, 6>;
using C3200 = RList<5, 5, 16, 8>;
using C3402 = RList<3, 9, 9, 14>;
using C3500 = RList<5, 7, 10, 10>;
using C3888 = RList<9, 12, 6, 6>;
using C4000 = RList<10, 10, 10, 4>;
using C4050 = RList<5, 9, 9, 10>;
using C4374 = RList<9, 9, 9, 6>;

// Alternative row kernels (opt-in, LL_KERNELS_ALT_WIDE): twice the warps per
// SM (64-80 registers, 3 CTAs of 8 or 10 warps) but every stage through
// shared memory.  Measured (ms/iter, alternative against default): 2048K
// 0.0435 / 0.0366, 3200K 0.0679 / 0.0629, 3136K 0.0643 / 0.0650, 1440K
// 0.0382 / 0.0418.
// Rows of 2048 (8x4x8x8) and 3072 (8x6x8x8) measured slower too: 12288K
// 0.2730 / 0.2560, 18432K 0.4102 / 0.3775; they are not compiled.
using A1280 = RList<8, 4, 5, 8>;  // 160 threads per row, 8 elements each
using A1024 = RList<8, 4, 4, 8>;
static const StaticWide kWide[] = {
    LLB_WIDE(L256, 4),  LLB_WIDE(L256, 2),  LLB_WIDE(L512, 4),  LLB_WIDE(L768, 4),  LLB_WIDE(L1024, 2), LLB_WIDE(L1280, 2),
    LLB_WIDE(L1536, 2), LLB_WIDE(L1792, 2), LLB_WIDE(L2048, 2), LLB_WIDE(L2304, 2),
    LLB_WIDE(L2560, 2), LLB_WIDE(L3072, 2), LLB_WIDE(L3584, 1), LLB_WIDE(L4096, 1),
    LLB_WIDE_ANY(A1280, 2, 3), LLB_WIDE_ANY(A1024, 2, 3),
};
// the row kernel variants a context may use: with LL_KERNELS_ALT_WIDE the
// alternative kernel of a length replaces the others of that length
static bool wide_allowed(const StaticWide &w, const ll_tuning *t) {
  const bool want_alt = t && (t->kernels & LL_KERNELS_ALT_WIDE);
  if (w.alt) return want_alt;
  if (!want_alt) return true;
  for (const auto &k : kWide)
    if (k.alt && k.L == w.L) return false;
  return true;
}
// Column lengths outside the 16 x M x 16 family that the length policy meets
// with a specialised row length: the fewest stages of radices <= 16, and the
// fewest threads per column that keep a stage's butterflies of one thread
// within 16 elements.  These lengths are short and their passes
// latency-bound, so a CTA takes one or two column pairs: about 128 CTAs at
// the row lengths they meet (256 for columns up to 252, 512 above), which
// spreads the loads over many SMs.
static const StaticTall kTall[] = {
    LLB_TALL(L256),  LLB_TALL(L512),  LLB_TALL(L768),  LLB_TALL(L1024), LLB_TALL(L1280), LLB_TALL(L1536), LLB_TALL(L1792),
    LLB_TALL(L2048), LLB_TALL(L2304), LLB_TALL(L2560), LLB_TALL(L3072), LLB_TALL(L3584), LLB_TALL(L4096),
    LLB_TALL_ANY(C24, 6, 1),        LLB_TALL_ANY(C28, 7, 1),
    LLB_TALL_ANY(C100, 10, 1),      LLB_TALL_ANY(C112, 8, 1),
    LLB_TALL_ANY(C120, 12, 1),      LLB_TALL_ANY(C128, 16, 2),
    LLB_TALL_ANY(C140, 14, 1),
    LLB_TALL_ANY(C160, 16, 1),      LLB_TALL_ANY(C168, 14, 1),
    LLB_TALL_ANY(C192, 16, 1),      LLB_TALL_ANY(C224, 16, 1),
    LLB_TALL_ANY(C240, 24, 1),      LLB_TALL_ANY(C252, 28, 1),
    LLB_TALL_ANY(C288, 32, 2),      LLB_TALL_ANY(C320, 32, 2),      LLB_TALL_ANY(C324, 81, 1),
    LLB_TALL_ANY(C336, 28, 2),      LLB_TALL_ANY(C360, 40, 2),
    LLB_TALL_ANY(C392, 28, 2),      LLB_TALL_ANY(C400, 40, 2),
    LLB_TALL_ANY(C448, 32, 2),      LLB_TALL_ANY(C576, 48, 2),
    LLB_TALL_ANY(C600, 60, 2),      LLB_TALL_ANY(C648, 72, 2),
    LLB_TALL_ANY(C672, 56, 2),      LLB_TALL_ANY(C720, 72, 2),
    LLB_TALL_ANY(C784, 56, 2),      LLB_TALL_ANY(C800, 80, 2),
    LLB_TALL_ANY(C1568, 112, 1),    LLB_TALL_ANY(C2744, 196, 1),
    LLB_TALL_ANY_SOLO(C1620, 180, 1),
    LLB_TALL_ANY_SOLO(C1728, 144, 1),
    LLB_TALL_ANY_SOLO(C1800, 150, 1),
    LLB_TALL_ANY_SOLO(C1944, 216, 1),
    LLB_TALL_ANY_SOLO(C2160, 180, 1),
    LLB_TALL_ANY_SOLO(C2240, 224, 1),
    LLB_TALL_ANY_SOLO(C2352, 196, 1),
    LLB_TALL_ANY_SOLO(C2400, 200, 1),
    LLB_TALL_ANY_SOLO(C2592, 216, 1),
    LLB_TALL_ANY_SOLO(C2688, 224, 1),
    LLB_TALL_ANY_SOLO(C2800, 200, 1),
    LLB_TALL_ANY_SOLO(C2880, 240, 1),
    LLB_TALL_ANY_SOLO(C2916, 324, 1),
    LLB_TALL_ANY_SOLO(C3024, 252, 1),
    LLB_TALL_ANY_SOLO(C3200, 214, 1),
    LLB_TALL_ANY_SOLO(C3402, 378, 1),
    LLB_TALL_ANY_SOLO(C3500, 350, 1),
    LLB_TALL_ANY_SOLO(C3888, 432, 1),
    LLB_TALL_ANY_SOLO(C4000, 400, 1),
    LLB_TALL_ANY_SOLO(C4050, 450, 1),
    LLB_TALL_ANY_SOLO(C4374, 486, 1),
};

// Fused cooperative kernels (fused_iters) for short lengths: the shape
// (row length W, column length H) they are compiled for.  The tall pass uses
// fewer column pairs per CTA than the two-launch kernels, for more CTAs.
struct FusedKernel {
  int W, H, G;  // G: rows per wide-pass unit (must equal the context's)
  void (*run)(TallArgs, WideArgs, uint32_t, int);
  int threads;      // per CTA
  int tall_ppc;     // column pairs per tall unit
  int smem;         // dynamic shared-memory entries
};
#define LLB_FUSED(LW, G, LT, TC, PP)                                                                        \
  {LW::L, LT::L, G, fused_iters<LW, G, FusedTall<LT, TC, PP>>, fused_threads<LW, G, FusedTall<LT, TC, PP>>(), \
   TC ? PP : 1,                                                                                              \
   std::max(G * row_slots<LW::L, G>() + tw_size<LW>(),                                                     \
            TC ? tall_any_smem<LT, PP>() : padded(2 * LT::L) + tall_extra<LT>())}
static const FusedKernel kFused[] = {
    LLB_FUSED(L256, 2, C24, 6, 8),
    LLB_FUSED(L256, 2, C28, 7, 16),
    LLB_FUSED(L256, 2, C112, 8, 4),
};
static const FusedKernel *find_fused(int W, int H, int G) {
  for (const auto &k : kFused)
    if (k.W == W && k.H == H && k.G == G) return &k;
  return nullptr;
}

// Cluster-resident kernels (cluster_iters) for short lengths: the shape
// (W, H), the row radix list and threads per row, the cluster size C and
// the launch.  Of the entries of a shape, the first whose cluster can be
// scheduled on the device is used (ll_tuning.cluster_variant picks another).
struct ClusterKernel {
  int W, H, C;
  void (*run)(TallArgs, WideArgs, const double2 *, uint32_t, int);
  int nrad, rad[4];    // row radix list
  int ncrad, crad[4];  // column radix list
  int tw;              // stage twiddle entries of both lists
  int threads;         // per CTA
  int smem;            // dynamic shared-memory entries
};
#define LLB_CRAD(LIST)                                                                                \
  LIST::N, {LIST::a[0], LIST::N > 1 ? LIST::a[1 % LIST::N] : 0, LIST::N > 2 ? LIST::a[2 % LIST::N] : 0, \
            LIST::N > 3 ? LIST::a[3 % LIST::N] : 0}
#define LLB_CLUSTER(PR, TWR, LT, TC, C, RPC)                                                                     \
  {PR::L, LT::L, C, cluster_iters<PR, TWR, LT, TC, C, RPC>, LLB_RAD(PR), LLB_CRAD(LT), tw_size<PR>() + tw_size<LT>(), \
   ClusterCfg<PR, TWR, LT, TC, C, RPC>::T, ClusterCfg<PR, TWR, LT, TC, C, RPC>::total}
// row lists of 256: 64 threads per row (one radix-4 butterfly each per
// stage) or 32 threads per row
using R256A = RList<4, 4, 4, 4>;
using R256B = RList<8, 4, 8>;
// rows of 768 and 1024: 192 and 256 threads per row (both directions run the
// list in the same order, so it need not be palindromic)
using R768 = RList<4, 6, 8, 4>;
using R1024 = RList<4, 8, 8, 4>;
using R768B = RList<8, 12, 8>;    // 96 threads per row
using R1024B = RList<8, 16, 8>;   // 128 threads per row
// column lists of small radices: many threads per column, short chains
using K16 = RList<4, 4>;
using K20 = RList<4, 5>;
using K24 = RList<4, 6>;
using K28 = RList<4, 7>;
using K32 = RList<4, 8>;
using K36 = RList<6, 6>;
using K40 = RList<5, 8>;
using K64 = RList<4, 4, 4>;
using K112 = RList<4, 4, 7>;
// Only lengths where one cluster (16 SMs) beats two launches over the whole
// GPU (us per iteration, cluster against two launches): 8K 3.6 / 13.4, 10K
// 5.1 / 15.6, 12K 4.8 / 9.9, 14K 5.7 / 10.0, 16K 4.8 / 17.2, 18K 6.1 / 17.7,
// 20K 6.5 / 16.3, 32K 7.8 / 16.5, 56K 13.1 / 14.8, and with rows of 768 and
// 1024: 36K 11.6 / 16.1, 42K 12.9 / 16.3, 48K 14.5 / 21.7.  At 50K (15.7 /
// 11.7) and 96K (21.7 / 12.1) the arithmetic of 16 SMs is the bound and the
// two-launch path stays.
static const ClusterKernel kCluster[] = {
    LLB_CLUSTER(R256A, 64, K16, 4, 16, 1),    LLB_CLUSTER(R256B, 32, K20, 5, 16, 2),
    LLB_CLUSTER(R256A, 64, K24, 6, 16, 2),    LLB_CLUSTER(R256B, 32, K24, 6, 16, 2),
    LLB_CLUSTER(R256A, 64, K24, 6, 8, 4),     LLB_CLUSTER(R256B, 32, K28, 7, 16, 2),
    LLB_CLUSTER(R256A, 64, K28, 7, 8, 4),     LLB_CLUSTER(R256A, 64, K32, 8, 16, 2),
    LLB_CLUSTER(R256B, 32, K36, 6, 16, 3),    LLB_CLUSTER(R256A, 64, K40, 8, 16, 4),
    LLB_CLUSTER(R256A, 64, K64, 16, 16, 4),   LLB_CLUSTER(R256B, 32, K112, 28, 16, 8),
    LLB_CLUSTER(R768, 192, K24, 6, 16, 2),    LLB_CLUSTER(R768B, 96, K24, 6, 16, 2),
    LLB_CLUSTER(R768B, 96, K28, 8, 16, 2),    LLB_CLUSTER(R768, 192, K28, 8, 16, 2),
    LLB_CLUSTER(R1024B, 128, K24, 6, 16, 2),  LLB_CLUSTER(R1024, 256, K24, 6, 16, 2),
};

static const StaticTall *find_tall(int L) {
  for (const auto &k : kTall)
    if (k.L == L) return &k;
  return nullptr;
}

}  // namespace llb

using namespace llb;

// ------------------------------------------------------------------ host --

namespace {

// e^{2 pi i num/den} rounded once from 80-bit arithmetic, with the angle
// reduced to the first octant so that cosl/sinl see small arguments.
double2 unit_root(unsigned long long num, unsigned long long den) {
  num %= den;
  // angle fraction f = num/den in [0,1); use 8*num relative to den for octant
  const long double PI = 3.14159265358979323846264338327950288L;
  unsigned long long n8 = num * 8;
  int oct = (int)(n8 / den);
  long double rem = (long double)(n8 - (unsigned long long)oct * den) / (long double)den;  // [0,1)
  long double a = rem * PI / 4;  // [0, pi/4)
  long double c, s;
  long double ca = cosl(a), sa = sinl(a), cb = cosl(PI / 4 - a), sb = sinl(PI / 4 - a);
  switch (oct) {
    case 0: c = ca; s = sa; break;
    case 1: c = sb; s = cb; break;
    case 2: c = -sa; s = ca; break;
    case 3: c = -cb; s = sb; break;
    case 4: c = -ca; s = -sa; break;
    case 5: c = -sb; s = -cb; break;
    case 6: c = sa; s = -ca; break;
    default: c = cb; s = -sb; break;
  }
  return make_double2((double)c, (double)s);
}

// Radices in the group order of fft_rows: 16, 8, 4, 2, 3, 5, 7.
bool make_plan(int L, FftPlan &p) {
  memset(&p, 0, sizeof(p));
  p.L = L;
  int m = L, k = 0;
  static const int rs[] = {16, 8, 4, 2, 3, 5, 7};
  for (int r : rs)
    while (m % r == 0) {
      if (k >= 10) return false;
      p.radix[k++] = r;
      m /= r;
    }
  p.nst = k;
  return m == 1;
}

bool seven_smooth(long long v) {
  if (v <= 0) return false;
  for (int p : {2, 3, 5, 7})
    while (v % p == 0) v /= p;
  return v == 1;
}

struct Shape {
  int W, H, G, T1, T2;
  const StaticWide *sw = nullptr;  // specialised kernels, when both exist
  const StaticTall *st = nullptr;
};

size_t wide_smem(int W, int G) { return sizeof(double2) * (size_t)padded(G * W); }
size_t tall_smem(int H) { return sizeof(double2) * (size_t)padded(2 * H); }
const size_t SMEM_MAX = 227 * 1024;

const int TMAX = 256;  // threads per CTA (128 registers per thread)

int round_threads(int need) {
  int t = (need + 31) / 32 * 32;
  return std::min(std::max(t, 64), TMAX);
}

bool shape_ok(long long N, int W, int G, Shape &s) {
  if (W < 16 || N % W) return false;
  long long H = N / W;
  if (W % 2 || H % 2 || H < 16) return false;
  if (H % G) return false;
  FftPlan p;
  if (!make_plan(W, p) || !make_plan((int)H, p)) return false;
  if (G * W > EPT * TMAX || H > EPT * TMAX) return false;
  if (wide_smem(W, G) > SMEM_MAX || tall_smem((int)H) > SMEM_MAX) return false;
  s.W = W;
  s.H = (int)H;
  s.G = G;
  s.T1 = round_threads((G * W + EPT - 1) / EPT);
  s.T2 = round_threads((int)((2 * H + EPT - 1) / EPT));
  return true;
}

// W near sqrt(N); G rows per wide-pass CTA such that a CTA's rows stay
// within ~100 KB of shared memory (two CTAs per SM).
// Of two rows-per-CTA counts G for one row length: the larger as long as it
// leaves at least 32 row groups (CTAs of the wide pass), else the smaller,
// so that short lengths spread their rows over more SMs.
static bool prefer_rows(long long H, int g, int cur) {
  const bool ok_g = H / g >= 32, ok_c = H / cur >= 32;
  if (ok_g != ok_c) return ok_g;
  return ok_g ? g > cur : g < cur;
}

bool choose_shape(long long N, const ll_tuning *t, Shape &out) {
  if (N % 2 || !seven_smooth(N)) return false;
  // compile-time specialised kernels for both passes, W closest to sqrt(N)
  if (!(t && (t->rows_per_cta > 0 || t->threads_wide > 0 || t->threads_tall > 0 || (t->kernels & LL_KERNELS_GENERIC)))) {
    const StaticWide *bw = nullptr;
    const StaticTall *bt = nullptr;
    double best = 1e30;
    for (const auto &w : kWide) {
      if (N % w.L || !wide_allowed(w, t)) continue;
      if (t && t->width > 0 && t->width != w.L) continue;
      const long long H = N / w.L;
      const StaticTall *tt = find_tall((int)H);
      if (!tt || H % w.G) continue;
      const double d = fabs(log((double)w.L / sqrt((double)N)));
      if (d < best || (d == best && bw && bw->L == w.L && prefer_rows(H, w.G, bw->G))) {
        best = d;
        bw = &w;
        bt = tt;
      }
    }
    if (bw) {
      out.W = bw->L;
      out.H = (int)(N / bw->L);
      out.G = bw->G;
      out.T1 = bw->G * bw->tr;
      out.T2 = bt->threads;
      out.sw = bw;
      out.st = bt;
      return true;
    }
    // a specialised wide pass with the generic tall pass, when the columns
    // have no specialised length (the wide pass is the costlier one)
    for (const auto &w : kWide) {
      if (N % w.L || !wide_allowed(w, t)) continue;
      if (t && t->width > 0 && t->width != w.L) continue;
      const long long H = N / w.L;
      Shape s;
      if (H % w.G || !shape_ok(N, w.L, w.G, s) || s.T2 > TMAX || s.H > EPT * s.T2) continue;
      const double d = fabs(log((double)w.L / sqrt((double)N)));
      if (d < best || (d == best && bw && bw->L == w.L && prefer_rows(H, w.G, bw->G))) {
        best = d;
        bw = &w;
        out = s;
      }
    }
    if (bw) {
      out.T1 = bw->G * bw->tr;
      out.sw = bw;
      out.st = nullptr;
      return true;
    }
  }
  std::vector<int> ws;
  if (t && t->width > 0) ws.push_back(t->width);
  else {
    for (long long w = 16; w <= 8192 && w <= N; w += 2)
      if (N % w == 0) ws.push_back((int)w);
    double root = sqrt((double)N);
    std::stable_sort(ws.begin(), ws.end(), [root](int a, int b) {
      return fabs(log((double)a / root)) < fabs(log((double)b / root));
    });
  }
  for (int w : ws) {
    std::vector<int> gs;
    if (t && t->rows_per_cta > 0) gs.push_back(t->rows_per_cta);
    else
      for (int g : {8, 4, 2, 1})
        if (wide_smem(w, g) <= 100 * 1024 || g == 1) gs.push_back(g);
    for (int g : gs) {
      Shape s;
      if (!shape_ok(N, w, g, s)) continue;
      if (t && t->threads_wide > 0) s.T1 = t->threads_wide;
      if (t && t->threads_tall > 0) s.T2 = t->threads_tall;
      if (s.T1 > TMAX || s.T2 > TMAX || s.T1 % 32 || s.T2 % 32 || s.G * s.W > EPT * s.T1 || s.H > EPT * s.T2)
        continue;
      out = s;
      return true;
    }
  }
  return false;
}

size_t shape_wide_smem(const Shape &s) {
  if (s.sw) return sizeof(double2) * (size_t)(s.sw->rows + s.sw->extra);
  return wide_smem(s.W, s.G);
}
size_t shape_tall_smem(const Shape &s) {
  return s.st ? sizeof(double2) * (size_t)s.st->smem : tall_smem(s.H);
}
// CTAs of the tall pass
int tall_grid(const Shape &s) { return s.st ? (s.W / 2 + s.st->ppc - 1) / s.st->ppc : s.W / 2; }

// Stage twiddles of a radix list in the order the specialised kernels read
// them: for each stage with NS > 1, rows k < NS of w_{NS*R}^(r*k), r = 1..R-1,
// each row padded to an odd length (tw_stride in kernels_static.cuh).
std::vector<double2> stage_twiddles(const int *rad, int nrad) {
  std::vector<double2> out;
  long long ns = 1;
  for (int i = 0; i < nrad; ++i) {
    const int R = rad[i];
    if (ns > 1)
      for (long long k = 0; k < ns; ++k) {
        for (int r = 1; r < R; ++r) out.push_back(unit_root((unsigned long long)(r * k), (unsigned long long)(ns * R)));
        if ((R - 1) % 2 == 0) out.push_back(make_double2(0.0, 0.0));
      }
    ns *= R;
  }
  return out;
}

}  // namespace

// Launch preferences measured on the B200 for lengths of the reference's
// table where the engine's default shape (row width nearest sqrt(N)) is not
// the fastest: the row width and ll_tuning.kernels to use when the caller
// gives no tuning.  A `<gpu> shapes.txt` from llucas -cufftbench, or any
// explicit tuning, takes precedence.
struct PreferredShape {
  uint32_t n;       // FFT length in words
  int32_t width;    // row width W
  int32_t kernels;  // LL_KERNELS_* flags
};
// (fftbench --all-shapes over the table lengths, 200 iterations timed with
// CUDA events; kept where the preference is at least 8 % faster)
static const PreferredShape kPreferred[] = {
    {288u * 1024, 256, 0},  // 288K: 0.0159 against 0.0220 ms/iter (W = 512)
    {324u * 1024, 256, 0},  // 324K: 0.0176 against 0.0227 ms/iter (W = 512)
    {336u * 1024, 768, 0},  // 336K: 0.0175 against 0.0243 ms/iter (W = 512)
    {360u * 1024, 768, 0},  // 360K: 0.0181 against 0.0254 ms/iter (W = 512)
    {392u * 1024, 256, 0},  // 392K: 0.0183 against 0.0255 ms/iter (W = 512)
    {400u * 1024, 256, 0},  // 400K: 0.0184 against 0.0255 ms/iter (W = 512)
    {448u * 1024, 1024, 0},  // 448K: 0.0181 against 0.0250 ms/iter (W = 512)
    {576u * 1024, 1536, 0},  // 576K: 0.0212 against 0.0270 ms/iter (W = 512)
    {640u * 1024, 256, 0},  // 640K: 0.0183 against 0.0308 ms/iter (W = 1024)
    {672u * 1024, 1792, 0},  // 672K: 0.0232 against 0.0293 ms/iter (W = 512)
    {768u * 1024, 256, 0},  // 768K: 0.0217 against 0.0248 ms/iter (W = 512)
    {784u * 1024, 1792, 0},  // 784K: 0.0264 against 0.0298 ms/iter (W = 512)
    {896u * 1024, 256, 0},  // 896K: 0.0223 against 0.0342 ms/iter (W = 1024)
    {1024u * 1024, 512, 0},  // 1024K: 0.0203 against 0.0249 ms/iter (W = 1024)
    {1280u * 1024, 256, 0},  // 1280K: 0.0285 against 0.0342 ms/iter (W = 1280)
    {1296u * 1024, 2304, 0},  // 1296K: 0.0292 against 0.0410 ms/iter (W = 1024)
    {1344u * 1024, 1024, 32},  // 1344K: 0.0322 against 0.0364 ms/iter (W = 1024)
    {1440u * 1024, 2560, 0},  // 1440K: 0.0334 against 0.0424 ms/iter (W = 1024)
    {1568u * 1024, 512, 0},  // 1568K: 0.0322 against 0.0373 ms/iter (W = 1024)
    {1600u * 1024, 1024, 32},  // 1600K: 0.0373 against 0.0417 ms/iter (W = 1024)
    {2160u * 1024, 512, 0},  // 2160K: 0.0474 against 0.0559 ms/iter (W = 1536)
    {2880u * 1024, 2560, 0},  // 2880K: 0.0626 against 0.0794 ms/iter (W = 2048)
    {3024u * 1024, 512, 0},  // 3024K: 0.0678 against 0.0768 ms/iter (W = 2304)
    {3600u * 1024, 2304, 0},  // 3600K: 0.0879 against 0.0968 ms/iter (W = 1024)
    {5120u * 1024, 1280, 0},  // 5120K: 0.0955 against 0.1032 ms/iter (W = 2048)
    {7200u * 1024, 1280, 0},  // 7200K: 0.1653 against 0.1885 ms/iter (W = 2048)
    {7776u * 1024, 1536, 0},  // 7776K: 0.1807 against 0.2043 ms/iter (W = 2048)
    {9216u * 1024, 1536, 0},  // 9216K: 0.1826 against 0.1994 ms/iter (W = 2048)
    {9408u * 1024, 3072, 0},  // 9408K: 0.2007 against 0.2243 ms/iter (W = 2048)
    {10240u * 1024, 1280, 0},  // 10240K: 0.1980 against 0.2223 ms/iter (W = 2048)
    {10800u * 1024, 2560, 0},  // 10800K: 0.2847 against 0.3449 ms/iter (W = 2304)
    {12288u * 1024, 3072, 0},  // 12288K: 0.2316 against 0.2559 ms/iter (W = 2048)
    {14336u * 1024, 1792, 0},  // 14336K: 0.2879 against 0.4295 ms/iter (W = 3584)
    {16384u * 1024, 2048, 0},  // 16384K: 0.3229 against 0.4005 ms/iter (W = 4096)
    {27216u * 1024, 4096, 0},  // 27216K: 0.8166 against 0.9911 ms/iter (W = 3584)
    {28000u * 1024, 4096, 0},  // 28000K: 0.8687 against 1.0280 ms/iter (W = 3584)
    {28672u * 1024, 4096, 0},  // 28672K: 0.7620 against 0.9017 ms/iter (W = 3584)
    {0, 0, 0},
};

static bool tuning_is_default(const ll_tuning *t) {
  return !t || (t->width == 0 && t->rows_per_cta == 0 && t->threads_wide == 0 && t->threads_tall == 0 &&
                t->kernels == 0 && t->cluster_variant == 0);
}

// The tuning a context of length n runs with: the caller's, or the measured
// preference for n when the caller leaves every choice to the engine.
static const ll_tuning *effective_tuning(uint32_t n, const ll_tuning *t, ll_tuning &store) {
  if (!tuning_is_default(t)) return t;
  for (const auto &p : kPreferred)
    if (p.n && p.n == n) {
      store = t ? *t : ll_tuning{};
      store.width = p.width;
      store.kernels = p.kernels;
      return &store;
    }
  return t;
}

struct ll_ctx {
  int device = 0;
  uint32_t q = 0, n = 0, b = 0, qn = 0;
  int N = 0;
  Shape shape{};
  FftPlan pw{}, ph{};
  int ts = 0;
  cudaStream_t stream = nullptr;
  // device buffers
  double2 *A = nullptr;
  int32_t *xint = nullptr;
  int32_t *ck_digits = nullptr;  // device-resident checkpoint (allocated on first use)
  uint32_t ck_offset = 0;
  bool ck_valid = false;
  long long *carry = nullptr;
  uint32_t *flags = nullptr;
  DevState *st = nullptr;
  double2 *twW = nullptr, *twH = nullptr, *thi = nullptr, *tlo = nullptr;
  double2 *stwW = nullptr, *stwH = nullptr;
  int32_t *rowE = nullptr, *colF = nullptr;
  double *rowW = nullptr, *rowWi = nullptr, *colW = nullptr, *colWi = nullptr;
  // host mirror
  uint32_t offset = 0;
  bool digits_current = false;
  bool started = false;
  int inject = 0;
  bool pdl = false;  // chain the passes with programmatic dependent launch
  const FusedKernel *fused = nullptr;  // iterations as one cooperative launch
  int fused_grid = 0;
  const ClusterKernel *cluster = nullptr;  // iterations as one cluster-resident launch
  double2 *stwC = nullptr;                 // stage twiddles of its row radix list
  float pending_err = 0.f;
  std::string err;
  TallArgs ta{};
  WideArgs wa{};
  // CUDA graph of `graph_iters` plain iterations, captured on first use
  int graph_iters = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

static ll_status cuda_fail(ll_ctx *c, cudaError_t e, const char *what) {
  if (c) {
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
  }
  return LL_ERR_CUDA;
}

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);       \
  } while (0)

template <typename T>
static cudaError_t upload(T **dst, const std::vector<T> &v) {
  cudaError_t e = cudaMalloc((void **)dst, sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice);
}

static void free_ctx(ll_ctx *c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  void *ptrs[] = {c->A, c->xint, c->ck_digits, c->carry, c->flags, c->st, c->twW, c->twH, c->thi, c->tlo, c->stwW, c->stwH, c->stwC,
                  c->rowE, c->colF, c->rowW, c->rowWi, c->colW, c->colWi};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  if (c->stream) cudaStreamDestroy(c->stream);
  cudaSetDevice(prev);
  delete c;
}

static ll_status build_tables(ll_ctx *ctx) {
  const int W = ctx->shape.W, H = ctx->shape.H, N = ctx->N;
  const uint32_t n = ctx->n, b = ctx->b;
  std::vector<double2> tw(W);
  for (int e = 0; e < W; ++e) tw[e] = unit_root(e, W);
  CK(upload(&ctx->twW, tw));
  tw.resize(H);
  for (int e = 0; e < H; ++e) tw[e] = unit_root(e, H);
  CK(upload(&ctx->twH, tw));
  int ts = 0;
  while ((1 << (ts + 1)) * (long long)(1 << (ts + 1)) <= (long long)N * 4 && ts < 14) ++ts;
  ctx->ts = ts;
  std::vector<double2> lo(1 << ts), hi((N >> ts) + 1);
  for (int e = 0; e < (1 << ts); ++e) lo[e] = unit_root(e, N);
  for (size_t e = 0; e < hi.size(); ++e) hi[e] = unit_root((unsigned long long)e << ts, N);
  CK(upload(&ctx->tlo, lo));
  CK(upload(&ctx->thi, hi));
  // weights: word j = 2H*m1 + (2*m2 + t); e_j = (rowE + colF) mod n
  const long double LN = (long double)n;
  std::vector<int32_t> rE(2 * H), cF(W);
  std::vector<double> rW(2 * H), rWi(2 * H), cW(W), cWi(W);
  for (int jr = 0; jr < 2 * H; ++jr) {
    long long e = (-(long long)jr * b) % (long long)n;
    if (e < 0) e += n;
    rE[jr] = (int32_t)e;
    rW[jr] = (double)exp2l((long double)e / LN);
    rWi[jr] = (double)(exp2l(-(long double)e / LN) / (long double)N);
  }
  for (int m1 = 0; m1 < W; ++m1) {
    long long e = (-((long long)2 * H * m1 % (long long)n) * (long long)b) % (long long)n;
    if (e < 0) e += n;
    cF[m1] = (int32_t)e;
    cW[m1] = (double)exp2l((long double)e / LN);
    cWi[m1] = (double)exp2l(-(long double)e / LN);
  }
  if (ctx->shape.sw) {
    std::vector<double2> t = stage_twiddles(ctx->shape.sw->rad, ctx->shape.sw->nrad);
    if ((int)t.size() != ctx->shape.sw->extra) return LL_ERR_SHAPE;
    CK(upload(&ctx->stwW, t));
  }
  if (ctx->shape.st) {
    std::vector<double2> t = stage_twiddles(ctx->shape.st->rad, ctx->shape.st->nrad);
    if ((int)t.size() != ctx->shape.st->tw) return LL_ERR_SHAPE;
    CK(upload(&ctx->stwH, t));
  }
  CK(upload(&ctx->rowE, rE));
  CK(upload(&ctx->rowW, rW));
  CK(upload(&ctx->rowWi, rWi));
  CK(upload(&ctx->colF, cF));
  CK(upload(&ctx->colW, cW));
  CK(upload(&ctx->colWi, cWi));
  return LL_OK;
}

extern "C" {

const char *ll_status_string(ll_status s) {
  switch (s) {
    case LL_OK: return "ok";
    case LL_ERR_ARG: return "invalid argument";
    case LL_ERR_SHAPE: return "unsupported FFT length";
    case LL_ERR_CUDA: return "CUDA error";
    case LL_ERR_NOMEM: return "out of memory";
    case LL_ERR_STATE: return "call out of order";
    case LL_ERR_TIMEOUT: return "device wait timed out";
    case LL_ERR_INJECTED: return "injected failure";
  }
  return "unknown status";
}

ll_status ll_create(int device, uint32_t q, uint32_t n, const ll_tuning *tuning, ll_ctx **out) {
  if (!out) return LL_ERR_ARG;
  *out = nullptr;
  if (n < 64 || n % 4 || q <= n || q > 0x7fffffffu || (q & 1) == 0) return LL_ERR_ARG;
  ll_tuning pref{};
  tuning = effective_tuning(n, tuning, pref);
  Shape s;
  if (!choose_shape((long long)n / 2, tuning, s)) return LL_ERR_SHAPE;
  ll_ctx *ctx = new ll_ctx();
  ctx->device = device;
  ctx->q = q;
  ctx->n = n;
  ctx->b = q % n;
  ctx->qn = q / n;
  ctx->N = (int)(n / 2);
  ctx->shape = s;
  ctx->graph_iters = tuning && tuning->graph_iters > 0 ? tuning->graph_iters : 64;
  if (tuning && tuning->graph_iters < 0) ctx->graph_iters = 0;  // graphs disabled
  if (ctx->qn + 1 > 30) { delete ctx; return LL_ERR_ARG; }
  make_plan(s.W, ctx->pw);
  make_plan(s.H, ctx->ph);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { delete ctx; return LL_ERR_CUDA; }
  ll_status rc = LL_OK;
  do {
    e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { rc = cuda_fail(ctx, e, "stream"); break; }
    const int ngroups = s.H / s.G;
    if ((e = cudaMalloc((void **)&ctx->A, sizeof(double2) * (size_t)ctx->N)) != cudaSuccess ||
        (e = cudaMalloc((void **)&ctx->xint, sizeof(int32_t) * (size_t)n)) != cudaSuccess ||
        (e = cudaMalloc((void **)&ctx->carry, sizeof(long long) * (size_t)ngroups * s.W)) != cudaSuccess ||
        (e = cudaMalloc((void **)&ctx->flags, sizeof(uint32_t) * kWarpFlags * (size_t)ngroups)) != cudaSuccess ||
        (e = cudaMalloc((void **)&ctx->st, sizeof(DevState))) != cudaSuccess) {
      rc = e == cudaErrorMemoryAllocation ? LL_ERR_NOMEM : cuda_fail(ctx, e, "cudaMalloc");
      break;
    }
    if ((e = cudaMemset(ctx->flags, 0, sizeof(uint32_t) * kWarpFlags * (size_t)ngroups)) != cudaSuccess ||
        (e = cudaMemset(ctx->st, 0, sizeof(DevState))) != cudaSuccess) {
      rc = cuda_fail(ctx, e, "cudaMemset");
      break;
    }
    rc = build_tables(ctx);
    if (rc != LL_OK) break;
    // The dynamic shared-memory limit is a per-function (not per-context)
    // attribute: raise it to the largest size any context has needed.
    {
      static std::mutex mu;
      static size_t max_sw = 0, max_st = 0;
      std::lock_guard<std::mutex> lock(mu);
      const size_t sw = std::max(max_sw, shape_wide_smem(s)), st = std::max(max_st, shape_tall_smem(s));
      if ((e = cudaFuncSetAttribute(wide_kernel<EPT, WIDE_ITER>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
          (e = cudaFuncSetAttribute(wide_kernel<EPT, WIDE_REPORT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
          (e = cudaFuncSetAttribute(wide_kernel<EPT, WIDE_INIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
          (e = cudaFuncSetAttribute(tall_kernel<EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st)) != cudaSuccess) {
        rc = cuda_fail(ctx, e, "cudaFuncSetAttribute");
        break;
      }
      for (const auto &k : kWide)
        if ((e = cudaFuncSetAttribute(k.iter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k.report, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k.init, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k.iter_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sw)) != cudaSuccess)
          break;
      for (const auto &k : kTall)
        if (e == cudaSuccess &&
            ((e = cudaFuncSetAttribute(k.run, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st)) != cudaSuccess ||
             (k.batch &&
              (e = cudaFuncSetAttribute(k.batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)st)) != cudaSuccess)))
          break;
      if (e != cudaSuccess) {
        rc = cuda_fail(ctx, e, "cudaFuncSetAttribute (static)");
        break;
      }
      max_sw = sw;
      max_st = st;
    }
    // Programmatic dependent launch pays when a pass runs in a few waves (the
    // next pass's prologue overlaps this one's drain); with many waves it
    // measured slower, so it is used only up to four waves per pass.
    if (s.sw && s.st) {
      int sms = 0, bw = 0, bt = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bw, s.sw->iter, s.T1, shape_wide_smem(s)) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, s.st->run, s.T2, shape_tall_smem(s)) == cudaSuccess &&
          bw > 0 && bt > 0) {
        const long long ww = ((long long)(s.H / s.G) + (long long)sms * bw - 1) / ((long long)sms * bw);
        const long long wt = ((long long)tall_grid(s) + (long long)sms * bt - 1) / ((long long)sms * bt);
        ctx->pdl = ww <= 4 && wt <= 4;
      }
    }
    // On request, short lengths with a fused kernel run their plain
    // iterations as one cooperative launch, when all its CTAs fit on the GPU
    // at once.
    if (s.sw && s.st && tuning && (tuning->kernels & LL_KERNELS_FUSED)) {
      const FusedKernel *f = find_fused(s.W, s.H, s.G);
      int sms = 0, per_sm = 0, coop = 0;
      if (f && cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) == cudaSuccess && coop &&
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
          cudaFuncSetAttribute(f->run, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(double2) * (size_t)f->smem)) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f->run, f->threads,
                                                        sizeof(double2) * (size_t)f->smem) == cudaSuccess) {
        const int units = std::max((s.W / 2 + f->tall_ppc - 1) / f->tall_ppc, s.H / s.G);
        if (per_sm > 0 && units <= sms * per_sm) {
          ctx->fused = f;
          ctx->fused_grid = units;
        }
      }
    }
    // Short lengths with a cluster-resident kernel run every step as one
    // launch of one thread-block cluster (the default; LL_KERNELS_CLUSTER8
    // keeps to clusters of at most 8 CTAs, LL_KERNELS_NO_CLUSTER turns it off).
    // (Not when the tuning asks for the generic kernels or their launch shape.)
    const bool want_generic = tuning && (tuning->rows_per_cta > 0 || tuning->threads_wide > 0 ||
                                         tuning->threads_tall > 0 || (tuning->kernels & LL_KERNELS_GENERIC));
    if (!ctx->fused && !want_generic && !(tuning && (tuning->kernels & LL_KERNELS_NO_CLUSTER))) {
      int cl_ok = 0;
      if (cudaDeviceGetAttribute(&cl_ok, cudaDevAttrClusterLaunch, device) != cudaSuccess) cl_ok = 0;
      int variant = 0;
      for (const auto &k : kCluster) {
        if (!cl_ok || k.W != s.W || k.H != s.H) continue;
        if (k.C > 8 && tuning && (tuning->kernels & LL_KERNELS_CLUSTER8)) continue;
        if (tuning && tuning->cluster_variant > 0 && variant++ != tuning->cluster_variant) continue;
        const size_t bytes = sizeof(double2) * (size_t)k.smem;
        if (cudaFuncSetAttribute(k.run, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess ||
            (k.C > 8 && cudaFuncSetAttribute(k.run, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
          cudaGetLastError();
          continue;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)k.C);
        cfg.blockDim = dim3((unsigned)k.threads);
        cfg.dynamicSmemBytes = bytes;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)k.C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)k.run, &cfg) != cudaSuccess) {
          cudaGetLastError();
          continue;
        }
        if (nclusters > 0) {
          ctx->cluster = &k;
          break;
        }
      }
      if (ctx->cluster) {
        std::vector<double2> t = stage_twiddles(ctx->cluster->rad, ctx->cluster->nrad);
        const std::vector<double2> tc = stage_twiddles(ctx->cluster->crad, ctx->cluster->ncrad);
        t.insert(t.end(), tc.begin(), tc.end());
        if ((int)t.size() != ctx->cluster->tw) { rc = LL_ERR_SHAPE; break; }
        if ((e = upload(&ctx->stwC, t)) != cudaSuccess) { rc = cuda_fail(ctx, e, "upload"); break; }
      }
    }
    TallArgs &ta = ctx->ta;
    ta.A = ctx->A; ta.stw = ctx->stwH; ta.twH = ctx->twH; ta.thi = ctx->thi; ta.tlo = ctx->tlo; ta.st = ctx->st;
    ta.ph = ctx->ph; ta.W = s.W; ta.H = s.H; ta.N = ctx->N; ta.ts = ctx->ts; ta.tmask = (1 << ctx->ts) - 1; ta.q = q;
    WideArgs &wa = ctx->wa;
    wa.A = ctx->A; wa.stw = ctx->stwW; wa.xint = ctx->xint; wa.carry = ctx->carry; wa.flags = ctx->flags; wa.twW = ctx->twW;
    wa.rowE = ctx->rowE; wa.rowW = ctx->rowW; wa.rowWi = ctx->rowWi;
    wa.colF = ctx->colF; wa.colW = ctx->colW; wa.colWi = ctx->colWi;
    wa.st = ctx->st; wa.pw = ctx->pw; wa.W = s.W; wa.H = s.H; wa.G = s.G; wa.ngroups = ngroups;
    wa.q = q; wa.n = n; wa.b = ctx->b; wa.qn = ctx->qn;
    // A state larger than half of L2 is read from HBM by every pass: each CTA
    // prefetches into L2 the unit about one wave ahead (the CTAs resident at
    // once), so that unit's loads hit L2.
    {
      int l2 = 0, sms = 0, bw = 0, bt = 0;
      const bool big = cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device) == cudaSuccess &&
                       16.0 * ctx->N > 0.5 * l2;
      if (big && s.sw && s.st && !(tuning && (tuning->kernels & LL_KERNELS_NO_PREFETCH)) &&
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bw, s.sw->iter, s.T1, shape_wide_smem(s)) == cudaSuccess &&
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, s.st->run, s.T2, shape_tall_smem(s)) == cudaSuccess) {
        if (s.W >= 2048) wa.pf = sms * bw;  // the kernels of shorter rows have no prefetch
        if (s.st->ppc == 1 && s.H >= 2048) ta.pf = sms * bt;
      }
    }
    if (s.sw) {
      // column m1 = t + r*TR: exponent colF[t] - D_r (mod n), D_r = r*TR*2H*b mod n
      const long long TR = s.sw->tr;
      for (int r = 0; r < 16; ++r) {
        const long long D = (long long)((unsigned __int128)r * TR * 2 * s.H % n * ctx->b % n);
        wa.colD[r] = (int)D;
        wa.colS[r] = (double)exp2l(-(long double)D / (long double)n);
        wa.colSi[r] = (double)exp2l((long double)D / (long double)n);
        wa.colS2[r] = 2.0 * wa.colS[r];
        wa.colSi2[r] = 0.5 * wa.colSi[r];
      }
    }
  } while (0);
  cudaSetDevice(prev);
  if (rc != LL_OK) {
    free_ctx(ctx);
    return rc;
  }
  *out = ctx;
  return LL_OK;
}

void ll_destroy(ll_ctx *ctx) { free_ctx(ctx); }

// Launches a specialised pass.  `chained`: the previous operation in the
// stream is the other pass, so the launch may use programmatic stream
// serialization (the kernel runs its prologue while that pass drains and
// waits in griddep_wait() before touching the state).
static void launch_static(const void *k, void *args, int grid, int threads, size_t smem, cudaStream_t st,
                          bool chained) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = chained ? 1 : 0;
  void *argv[] = {args};
  cudaLaunchKernelExC(&cfg, k, argv);
}

static void launch_wide(ll_ctx *ctx, int mode, bool chained = false) {
  const Shape &s = ctx->shape;
  const size_t sm = shape_wide_smem(s);
  if (s.sw) {
    void (*k)(WideArgs) = mode == WIDE_INIT ? s.sw->init : mode == WIDE_REPORT ? s.sw->report : s.sw->iter;
    launch_static((const void *)k, &ctx->wa, s.H / s.G, s.T1, sm, ctx->stream, chained && ctx->pdl);
  } else if (mode == WIDE_INIT) {
    wide_kernel<EPT, WIDE_INIT><<<s.H / s.G, s.T1, sm, ctx->stream>>>(ctx->wa);
  } else if (mode == WIDE_REPORT) {
    wide_kernel<EPT, WIDE_REPORT><<<s.H / s.G, s.T1, sm, ctx->stream>>>(ctx->wa);
  } else {
    wide_kernel<EPT, WIDE_ITER><<<s.H / s.G, s.T1, sm, ctx->stream>>>(ctx->wa);
  }
}

static void launch_tall(ll_ctx *ctx, bool chained = false) {
  const Shape &s = ctx->shape;
  if (s.st) launch_static((const void *)s.st->run, &ctx->ta, tall_grid(s), s.T2, shape_tall_smem(s), ctx->stream, chained && ctx->pdl);
  else tall_kernel<EPT><<<s.W / 2, s.T2, tall_smem(s.H), ctx->stream>>>(ctx->ta);
}

static ll_status launch_init(ll_ctx *ctx) {
  launch_wide(ctx, WIDE_INIT);
  CK(cudaGetLastError());
  return LL_OK;
}

ll_status ll_load_digits(ll_ctx *ctx, const int32_t *digits, uint32_t offset) {
  if (!ctx || !digits || offset >= ctx->q) return LL_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->xint, digits, sizeof(int32_t) * ctx->n, cudaMemcpyHostToDevice, ctx->stream));
  DevState hs{};
  // keep the ticket counter: read it back so that the whole struct can be rewritten
  CK(cudaMemcpyAsync(&hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  hs.offset = offset;
  hs.err_bits = 0;
  hs.fault = 0;
  CK(cudaMemcpyAsync(ctx->st, &hs, sizeof(DevState), cudaMemcpyHostToDevice, ctx->stream));
  ll_status rc = launch_init(ctx);
  if (rc != LL_OK) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->offset = offset;
  ctx->digits_current = true;
  ctx->started = true;
  return LL_OK;
}

ll_status ll_start(ll_ctx *ctx, uint32_t offset) {
  if (!ctx || offset >= ctx->q) return LL_ERR_ARG;
  std::vector<int32_t> d(ctx->n, 0);
  const uint32_t pos = (offset + 2) % ctx->q;
  const uint32_t w = (uint32_t)(((unsigned long long)pos * ctx->n) / ctx->q);
  const uint32_t sw = (uint32_t)(((unsigned long long)w * ctx->q + ctx->n - 1) / ctx->n);
  d[w] = 1 << (pos - sw);
  return ll_load_digits(ctx, d.data(), offset);
}

static ll_status launch_iteration(ll_ctx *ctx, bool report) {
  launch_tall(ctx);
  launch_wide(ctx, report ? WIDE_REPORT : WIDE_ITER, true);
  CK(cudaGetLastError());
  ctx->offset = (uint32_t)((2ull * ctx->offset) % ctx->q);
  return LL_OK;
}

// Plain iterations as fused cooperative launches (at most 4096 per launch).
static ll_status launch_fused(ll_ctx *ctx, uint32_t iters) {
  const FusedKernel *f = ctx->fused;
  const Shape &s = ctx->shape;
  int tall_units = (s.W / 2 + f->tall_ppc - 1) / f->tall_ppc;
  for (uint32_t done = 0; done < iters;) {
    uint32_t k = std::min<uint32_t>(iters - done, 4096u);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctx->fused_grid);
    cfg.blockDim = dim3((unsigned)f->threads);
    cfg.dynamicSmemBytes = sizeof(double2) * (size_t)f->smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *argv[] = {(void *)&ctx->ta, (void *)&ctx->wa, (void *)&k, (void *)&tall_units};
    CK(cudaLaunchKernelExC(&cfg, (const void *)f->run, argv));
    for (uint32_t i = 0; i < k; ++i) ctx->offset = (uint32_t)((2ull * ctx->offset) % ctx->q);
    done += k;
  }
  return LL_OK;
}

// Iterations as cluster-resident launches (at most 65536 per launch, a
// fraction of a second at the lengths that have such a kernel); the last
// launch writes the digits when the step reports.
static ll_status launch_cluster(ll_ctx *ctx, uint32_t iters, bool report) {
  const ClusterKernel *f = ctx->cluster;
  for (uint32_t done = 0; done < iters;) {
    uint32_t k = std::min<uint32_t>(iters - done, 65536u);
    int rep = report && done + k == iters ? 1 : 0;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)f->C);
    cfg.blockDim = dim3((unsigned)f->threads);
    cfg.dynamicSmemBytes = sizeof(double2) * (size_t)f->smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)f->C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const double2 *stw = ctx->stwC;
    void *argv[] = {(void *)&ctx->ta, (void *)&ctx->wa, (void *)&stw, (void *)&k, (void *)&rep};
    CK(cudaLaunchKernelExC(&cfg, (const void *)f->run, argv));
    for (uint32_t i = 0; i < k; ++i) ctx->offset = (uint32_t)((2ull * ctx->offset) % ctx->q);
    done += k;
  }
  return LL_OK;
}

ll_status ll_step(ll_ctx *ctx, uint32_t iters, uint32_t flags, float *max_err) {
  if (!ctx) return LL_ERR_ARG;
  if (!ctx->started) return LL_ERR_STATE;
  if (ctx->inject > 0) {
    --ctx->inject;
    ctx->err = "injected failure";
    return LL_ERR_INJECTED;
  }
  CK(cudaSetDevice(ctx->device));
  const bool report = (flags & LL_REPORT) != 0;
  uint32_t done = 0;
  const uint32_t K = (uint32_t)ctx->graph_iters;
  if (ctx->cluster && iters) {
    const ll_status rc = launch_cluster(ctx, iters, report);
    if (rc != LL_OK) return rc;
    done = iters;
  } else if (ctx->fused && iters >= 2u + (report ? 1u : 0u)) {
    // plain iterations fused; the report iteration (if any) as two passes
    const uint32_t plain = iters - (report ? 1u : 0u);
    const ll_status rc = launch_fused(ctx, plain);
    if (rc != LL_OK) return rc;
    done = plain;
  } else if (K && iters >= K + (report ? 1u : 0u)) {
    // iterations without a report, K at a time, replayed from one CUDA graph
    if (!ctx->graph_exec) {
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      const uint32_t off0 = ctx->offset;
      for (uint32_t i = 0; i < K; ++i) {
        launch_tall(ctx, i > 0);
        launch_wide(ctx, WIDE_ITER, true);
      }
      ctx->offset = off0;
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &ctx->graph);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
      CK(cudaGraphInstantiate(&ctx->graph_exec, ctx->graph, 0));
    }
    const uint32_t plain = iters - (report ? 1u : 0u);
    while (plain - done >= K) {
      CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
      for (uint32_t i = 0; i < K; ++i) ctx->offset = (uint32_t)((2ull * ctx->offset) % ctx->q);
      done += K;
    }
  }
  for (uint32_t i = done; i < iters; ++i) {
    ll_status rc = launch_iteration(ctx, report && i + 1 == iters);
    if (rc != LL_OK) return rc;
  }
  if (iters) ctx->digits_current = report;
  if ((flags & (LL_REPORT | LL_ERRCHK)) && !(flags & LL_ASYNC)) {
    DevState hs{};
    CK(cudaMemcpyAsync(&hs, ctx->st, sizeof(DevState), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const uint32_t zero[2] = {0, 0};
    CK(cudaMemcpyAsync(&ctx->st->err_bits, zero, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    float e;
    memcpy(&e, &hs.err_bits, sizeof(float));
    if (max_err) *max_err = e;
    if (hs.offset != ctx->offset) {
      ctx->err = "device offset diverged from host mirror";
      return LL_ERR_STATE;
    }
    if (hs.fault & 1u) {
      ctx->err = "wide pass: carry wait timed out";
      return LL_ERR_TIMEOUT;
    }
    if (hs.fault & 2u) {
      ctx->err = "wide pass: a word beyond the exact FP64 range (roundoff far above 0.5, or digits out of range)";
      if (max_err) *max_err = 1.0f;
    }
  }
  return LL_OK;
}

ll_status ll_device_checkpoint(ll_ctx *ctx) {
  if (!ctx) return LL_ERR_ARG;
  if (!ctx->digits_current) return LL_ERR_STATE;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->ck_digits) {
    const cudaError_t e = cudaMalloc((void **)&ctx->ck_digits, sizeof(int32_t) * ctx->n);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? LL_ERR_NOMEM : cuda_fail(ctx, e, "cudaMalloc");
  }
  CK(cudaMemcpyAsync(ctx->ck_digits, ctx->xint, sizeof(int32_t) * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
  ctx->ck_offset = ctx->offset;
  ctx->ck_valid = true;
  return LL_OK;
}

ll_status ll_device_restore(ll_ctx *ctx, uint32_t *offset) {
  if (!ctx) return LL_ERR_ARG;
  if (!ctx->ck_valid) return LL_ERR_STATE;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(ctx->xint, ctx->ck_digits, sizeof(int32_t) * ctx->n, cudaMemcpyDeviceToDevice, ctx->stream));
  // offset, roundoff maximum and fault bits; the ticket counter is kept
  const uint32_t f[3] = {ctx->ck_offset, 0u, 0u};
  static_assert(offsetof(DevState, err_bits) == offsetof(DevState, offset) + 4 &&
                    offsetof(DevState, fault) == offsetof(DevState, offset) + 8,
                "offset, err_bits and fault are contiguous");
  CK(cudaMemcpyAsync(&ctx->st->offset, f, sizeof f, cudaMemcpyHostToDevice, ctx->stream));
  const ll_status rc = launch_init(ctx);
  if (rc != LL_OK) return rc;
  ctx->offset = ctx->ck_offset;
  ctx->digits_current = true;
  ctx->started = true;
  if (offset) *offset = ctx->offset;
  return LL_OK;
}

uint64_t ll_context_bytes(uint32_t q, uint32_t n, const ll_tuning *tuning) {
  ll_tuning pref{};
  tuning = effective_tuning(n, tuning, pref);
  Shape s;
  if (n < 64 || n % 4 || !choose_shape((long long)n / 2, tuning, s)) return 0;
  (void)q;
  const uint64_t N = n / 2, W = (uint64_t)s.W, H = (uint64_t)s.H, ng = (uint64_t)(s.H / s.G);
  int ts = 0;
  while ((1 << (ts + 1)) * (long long)(1 << (ts + 1)) <= (long long)N * 4 && ts < 14) ++ts;
  uint64_t b = 16 * N + 4ull * n + 8 * ng * W + 4 * kWarpFlags * ng + sizeof(DevState);  // state, digits, carries
  b += 16 * (W + H) + 16 * (((uint64_t)1 << ts) + (N >> ts) + 1);                     // twiddles
  b += 20 * 2 * H + 20 * W;                                                           // weights
  if (s.sw) b += 16 * (uint64_t)s.sw->extra;
  if (s.st) b += 16 * (uint64_t)s.st->tw;
  // the cluster kernel's stage twiddles, when the length has one (the
  // largest table among its variants)
  uint64_t tw_cluster = 0;
  for (const auto &k : kCluster)
    if (k.W == s.W && k.H == s.H) tw_cluster = std::max<uint64_t>(tw_cluster, 16 * (uint64_t)k.tw);
  b += tw_cluster;
  return b;
}

int32_t ll_busy(ll_ctx *ctx) {
  if (!ctx) return -1;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return -1;
  const cudaError_t e = cudaStreamQuery(ctx->stream);
  if (e == cudaSuccess) return 0;
  if (e == cudaErrorNotReady) return 1;
  ctx->err = cudaGetErrorString(e);
  return -1;
}

ll_status ll_sync(ll_ctx *ctx) {
  if (!ctx) return LL_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return LL_OK;
}

ll_status ll_read_digits(ll_ctx *ctx, int32_t *digits, uint32_t *offset) {
  if (!ctx || !digits) return LL_ERR_ARG;
  if (!ctx->digits_current) return LL_ERR_STATE;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(digits, ctx->xint, sizeof(int32_t) * ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (offset) *offset = ctx->offset;
  return LL_OK;
}

ll_status ll_res64(ll_ctx *ctx, uint64_t *res64) {
  if (!ctx || !res64) return LL_ERR_ARG;
  std::vector<int32_t> d(ctx->n);
  uint32_t off = 0;
  ll_status rc = ll_read_digits(ctx, d.data(), &off);
  if (rc != LL_OK) return rc;
  *res64 = ll_digits_res64(d.data(), ctx->q, ctx->n, off);
  return LL_OK;
}

uint32_t ll_exponent(const ll_ctx *ctx) { return ctx ? ctx->q : 0; }
uint32_t ll_fft_length(const ll_ctx *ctx) { return ctx ? ctx->n : 0; }
uint32_t ll_offset(const ll_ctx *ctx) { return ctx ? ctx->offset : 0; }
void *ll_stream(const ll_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
void ll_shape(const ll_ctx *ctx, int32_t *width, int32_t *height, int32_t *rows_per_cta, int32_t *threads_wide,
              int32_t *threads_tall) {
  if (!ctx) return;
  if (width) *width = ctx->shape.W;
  if (height) *height = ctx->shape.H;
  if (rows_per_cta) *rows_per_cta = ctx->shape.G;
  if (threads_wide) *threads_wide = ctx->shape.T1;
  if (threads_tall) *threads_tall = ctx->shape.T2;
}
const char *ll_last_error(const ll_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }
int32_t ll_check_tables(void) {
  int32_t bad = 0;
  for (const auto &p : kPreferred) {
    if (!p.n) continue;
    ll_tuning t{};
    t.width = p.width;
    t.kernels = p.kernels;
    Shape s;
    if (!choose_shape((long long)p.n / 2, &t, s) || s.W != p.width || !s.sw || !s.st) ++bad;
  }
  for (const auto &k : kWide)
    if ((int)stage_twiddles(k.rad, k.nrad).size() != k.extra) ++bad;
  for (const auto &k : kTall)
    if ((int)stage_twiddles(k.rad, k.nrad).size() != k.tw) ++bad;
  for (const auto &k : kCluster) {
    int L = 1, Lc = 1;
    for (int i = 0; i < k.nrad; ++i) L *= k.rad[i];
    for (int i = 0; i < k.ncrad; ++i) Lc *= k.crad[i];
    if (L != k.W || Lc != k.H ||
        (int)(stage_twiddles(k.rad, k.nrad).size() + stage_twiddles(k.crad, k.ncrad).size()) != k.tw)
      ++bad;
  }
  return bad;
}

int32_t ll_kernel_kinds(const ll_ctx *ctx) {
  if (!ctx) return 0;
  return (ctx->shape.sw ? 1 : 0) | (ctx->shape.st ? 2 : 0) | (ctx->fused ? 4 : 0) | (ctx->cluster ? 8 : 0);
}
void ll_debug_inject_failure(ll_ctx *ctx, int32_t count) {
  if (ctx) ctx->inject = count;
}

ll_status ll_debug_launch(ll_ctx *ctx, int32_t which) {
  if (!ctx || !ctx->started) return LL_ERR_STATE;
  CK(cudaSetDevice(ctx->device));
  if (which == 0) {
    launch_tall(ctx);
    ctx->offset = (uint32_t)((2ull * ctx->offset) % ctx->q);
  } else {
    launch_wide(ctx, WIDE_ITER);
  }
  ctx->digits_current = false;
  CK(cudaGetLastError());
  return LL_OK;
}

int32_t ll_device_name(int device, char *name, size_t len) {
  if (!name || !len) return -1;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return -1;
  snprintf(name, len, "%s", p.name);
  return 0;
}

int32_t ll_length_supported(uint32_t n) {
  if (n < 64 || n % 4) return 0;
  Shape s;
  return choose_shape((long long)n / 2, nullptr, s) ? 1 : 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or
// arena that owns all device memory, plugins whose host forbids allocation
// during a work call, and latency-critical loops that must not hit the
// allocator.  ll_step_static runs the same tall/wide kernels as ll_step, but
// every piece of device scratch -- the transform array, the carry hand-off
// rows, the ready flags, the device state and all tables -- is carved out of
// one file-scope __device__ array of LL_STATIC_SCRATCH_BYTES bytes.  Every GPU
// that loads this library holds that array until the process exits.
namespace {
constexpr size_t kScratchBytes = LL_STATIC_SCRATCH_BYTES;
}
static __device__ __align__(256) unsigned char g_ll_scratch[kScratchBytes];

namespace {

// Host-side table staging, also file-scope so that no call allocates.  It is
// guarded by g_table_mu only while the tables are built and copied: a copy
// from pageable host memory has consumed its source when cudaMemcpyAsync
// returns.  Each device's scratch is guarded by that device's own mutex, held
// until the call's work on the GPU has finished, so calls on different GPUs
// do not wait for each other's kernels.
constexpr int kMaxDevices = 64;
constexpr size_t kHostTableBytes = 2u << 20;
alignas(256) unsigned char g_host_tables[kHostTableBytes];
std::mutex g_table_mu;
std::mutex g_device_mu[kMaxDevices];
void *g_scratch_ptr[kMaxDevices] = {nullptr};  // device address of g_ll_scratch, per device

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Raises (never lowers) a kernel's dynamic shared-memory limit.
cudaError_t raise_smem_limit(const void *k, size_t bytes) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, k);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

extern "C" ll_status ll_step_static(int device, uint32_t q, uint32_t n, uint32_t offset, uint32_t iters,
                                    const int32_t *digits_in, int32_t *digits_out, float *max_err,
                                    void *stream) {
  if (!digits_in || !digits_out || n < 64 || n % 4 || q <= n || (q & 1) == 0 || offset >= q) return LL_ERR_ARG;
  if (n > LL_STATIC_MAX_WORDS) return LL_ERR_ARG;  // beyond the static scratch's stated maximum
  if (device < 0 || device >= kMaxDevices) return LL_ERR_ARG;
  const int N = (int)(n / 2);
  Shape s;
  if (!choose_shape(N, nullptr, s)) return LL_ERR_SHAPE;
  std::lock_guard<std::mutex> lock(g_device_mu[device]);
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return LL_ERR_CUDA;
  cudaStream_t st = (cudaStream_t)stream;
  // Declared after the lock, so destroyed before it: on every return, work
  // this call has enqueued finishes before another call may reuse the
  // scratch, and the caller's current device is put back.
  struct Restore {
    int d;
    cudaStream_t s;
    bool enqueued = false;
    ~Restore() {
      if (enqueued) cudaStreamSynchronize(s);
      cudaSetDevice(d);
    }
  } restore{prev, st};
  std::unique_lock<std::mutex> table_lock(g_table_mu);
  // set-up, once per device: the device address of the static array
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_ll_scratch) != cudaSuccess || !p) return LL_ERR_CUDA;
    g_scratch_ptr[device] = p;
  }
  unsigned char *base = (unsigned char *)g_scratch_ptr[device];

  // ---- host tables (same definitions as build_tables) into the static staging
  const int W = s.W, H = s.H;
  const uint32_t b = q % n, qn = q / n;
  int ts = 0;
  while ((1 << (ts + 1)) * (long long)(1 << (ts + 1)) <= (long long)N * 4 && ts < 14) ++ts;
  const size_t n_lo = (size_t)1 << ts, n_hi = (size_t)(N >> ts) + 1;
  size_t ho = 0;
  auto hput = [&](size_t bytes) -> unsigned char * {
    unsigned char *p = g_host_tables + ho;
    ho = align256(ho + bytes);
    return ho <= kHostTableBytes ? p : nullptr;
  };
  double2 *h_twW = (double2 *)hput(sizeof(double2) * W);
  double2 *h_twH = (double2 *)hput(sizeof(double2) * H);
  double2 *h_lo = (double2 *)hput(sizeof(double2) * n_lo);
  double2 *h_hi = (double2 *)hput(sizeof(double2) * n_hi);
  int32_t *h_rE = (int32_t *)hput(sizeof(int32_t) * 2 * H);
  double *h_rW = (double *)hput(sizeof(double) * 2 * H);
  double *h_rWi = (double *)hput(sizeof(double) * 2 * H);
  int32_t *h_cF = (int32_t *)hput(sizeof(int32_t) * W);
  double *h_cW = (double *)hput(sizeof(double) * W);
  double *h_cWi = (double *)hput(sizeof(double) * W);
  const size_t n_stwW = s.sw ? (size_t)s.sw->extra : 0, n_stwH = s.st ? (size_t)s.st->tw : 0;
  double2 *h_stwW = (double2 *)hput(sizeof(double2) * (n_stwW ? n_stwW : 1));
  double2 *h_stwH = (double2 *)hput(sizeof(double2) * (n_stwH ? n_stwH : 1));
  if (!h_stwH) return LL_ERR_ARG;
  const size_t table_bytes = ho;
  for (int e = 0; e < W; ++e) h_twW[e] = unit_root(e, W);
  for (int e = 0; e < H; ++e) h_twH[e] = unit_root(e, H);
  for (size_t e = 0; e < n_lo; ++e) h_lo[e] = unit_root(e, N);
  for (size_t e = 0; e < n_hi; ++e) h_hi[e] = unit_root((unsigned long long)e << ts, N);
  const long double LN = (long double)n;
  for (int jr = 0; jr < 2 * H; ++jr) {
    long long e = (-(long long)jr * b) % (long long)n;
    if (e < 0) e += n;
    h_rE[jr] = (int32_t)e;
    h_rW[jr] = (double)exp2l((long double)e / LN);
    h_rWi[jr] = (double)(exp2l(-(long double)e / LN) / (long double)N);
  }
  for (int m1 = 0; m1 < W; ++m1) {
    long long e = (-((long long)2 * H * m1 % (long long)n) * (long long)b) % (long long)n;
    if (e < 0) e += n;
    h_cF[m1] = (int32_t)e;
    h_cW[m1] = (double)exp2l((long double)e / LN);
    h_cWi[m1] = (double)exp2l(-(long double)e / LN);
  }
  auto fill_stw = [](double2 *out, const int *rad, int nrad) {
    size_t k = 0;
    long long ns = 1;
    for (int i = 0; i < nrad; ++i) {
      const int R = rad[i];
      if (ns > 1)
        for (long long kk = 0; kk < ns; ++kk)
        {
          for (int r = 1; r < R; ++r) out[k++] = unit_root((unsigned long long)(r * kk), (unsigned long long)(ns * R));
          if ((R - 1) % 2 == 0) out[k++] = make_double2(0.0, 0.0);  // odd row stride (bank spread)
        }
      ns *= R;
    }
    return k;
  };
  if (s.sw && fill_stw(h_stwW, s.sw->rad, s.sw->nrad) != n_stwW) return LL_ERR_SHAPE;
  if (s.st && fill_stw(h_stwH, s.st->rad, s.st->nrad) != n_stwH) return LL_ERR_SHAPE;

  // ---- device carve-up of the static scratch
  const int ngroups = H / s.G;
  size_t o = 0;
  auto dput = [&](size_t bytes) -> unsigned char * {
    unsigned char *p = base + o;
    o = align256(o + bytes);
    return p;
  };
  double2 *A = (double2 *)dput(sizeof(double2) * (size_t)N);
  long long *carry = (long long *)dput(sizeof(long long) * (size_t)ngroups * W);
  uint32_t *flags = (uint32_t *)dput(sizeof(uint32_t) * kWarpFlags * (size_t)ngroups);
  DevState *dst = (DevState *)dput(sizeof(DevState));
  unsigned char *dtab = dput(table_bytes);
  if (o > kScratchBytes) return LL_ERR_ARG;  // shape needs more scratch than the static array holds
  auto dev = [&](const void *hp) { return dtab + ((const unsigned char *)hp - g_host_tables); };

  // ---- kernels' limits (raised only), arguments
  const size_t sw_bytes = shape_wide_smem(s), st_bytes = shape_tall_smem(s);
  cudaError_t e = cudaSuccess;
  if (s.sw) {
    if ((e = raise_smem_limit((const void *)s.sw->iter, sw_bytes)) != cudaSuccess ||
        (e = raise_smem_limit((const void *)s.sw->report, sw_bytes)) != cudaSuccess ||
        (e = raise_smem_limit((const void *)s.sw->init, sw_bytes)) != cudaSuccess)
      return LL_ERR_CUDA;
  } else if ((e = raise_smem_limit((const void *)wide_kernel<EPT, WIDE_ITER>, sw_bytes)) != cudaSuccess ||
             (e = raise_smem_limit((const void *)wide_kernel<EPT, WIDE_REPORT>, sw_bytes)) != cudaSuccess ||
             (e = raise_smem_limit((const void *)wide_kernel<EPT, WIDE_INIT>, sw_bytes)) != cudaSuccess) {
    return LL_ERR_CUDA;
  }
  if ((e = raise_smem_limit(s.st ? (const void *)s.st->run : (const void *)tall_kernel<EPT>, st_bytes)) !=
      cudaSuccess)
    return LL_ERR_CUDA;
  FftPlan pw, ph;
  make_plan(W, pw);
  make_plan(H, ph);
  TallArgs ta{};
  ta.A = A; ta.stw = (const double2 *)dev(h_stwH); ta.twH = (const double2 *)dev(h_twH);
  ta.thi = (const double2 *)dev(h_hi); ta.tlo = (const double2 *)dev(h_lo); ta.st = dst;
  ta.ph = ph; ta.W = W; ta.H = H; ta.N = N; ta.ts = ts; ta.tmask = (1 << ts) - 1; ta.q = q;
  WideArgs wa{};
  wa.A = A; wa.stw = (const double2 *)dev(h_stwW); wa.carry = carry; wa.flags = flags;
  wa.twW = (const double2 *)dev(h_twW);
  wa.rowE = (const int32_t *)dev(h_rE); wa.rowW = (const double *)dev(h_rW); wa.rowWi = (const double *)dev(h_rWi);
  wa.colF = (const int32_t *)dev(h_cF); wa.colW = (const double *)dev(h_cW); wa.colWi = (const double *)dev(h_cWi);
  wa.st = dst; wa.pw = pw; wa.W = W; wa.H = H; wa.G = s.G; wa.ngroups = ngroups;
  wa.q = q; wa.n = n; wa.b = b; wa.qn = qn;
  if (s.sw) {
    const long long TR = s.sw->tr;
    for (int r = 0; r < 16; ++r) {
      const long long D = (long long)((unsigned __int128)r * TR * 2 * H % n * b % n);
      wa.colD[r] = (int)D;
      wa.colS[r] = (double)exp2l(-(long double)D / (long double)n);
      wa.colSi[r] = (double)exp2l((long double)D / (long double)n);
      wa.colS2[r] = 2.0 * wa.colS[r];
      wa.colSi2[r] = 0.5 * wa.colSi[r];
    }
  }

  // ---- state that must start at zero: flags, ticket, error, fault
  DevState hs{};
  hs.offset = offset;
  restore.enqueued = true;
  if ((e = cudaMemsetAsync(flags, 0, sizeof(uint32_t) * kWarpFlags * (size_t)ngroups, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dst, &hs, sizeof(DevState), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dtab, g_host_tables, table_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return LL_ERR_CUDA;
  table_lock.unlock();  // the pageable-source copies above have consumed the host tables

  // ---- digits in -> weighted transform -> iters iterations -> digits out
  const dim3 gw(H / s.G), gt(tall_grid(s));
  wa.xint = const_cast<int32_t *>(digits_in);
  if (s.sw) s.sw->init<<<gw, s.T1, sw_bytes, st>>>(wa);
  else wide_kernel<EPT, WIDE_INIT><<<gw, s.T1, sw_bytes, st>>>(wa);
  if (iters == 0) {
    e = cudaMemcpyAsync(digits_out, digits_in, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return LL_ERR_CUDA;
  }
  for (uint32_t i = 0; i < iters; ++i) {
    if (s.st) s.st->run<<<gt, s.T2, st_bytes, st>>>(ta);
    else tall_kernel<EPT><<<gt, s.T2, st_bytes, st>>>(ta);
    const bool last = i + 1 == iters;
    wa.xint = last ? digits_out : nullptr;
    if (s.sw) (last ? s.sw->report : s.sw->iter)<<<gw, s.T1, sw_bytes, st>>>(wa);
    else if (last) wide_kernel<EPT, WIDE_REPORT><<<gw, s.T1, sw_bytes, st>>>(wa);
    else wide_kernel<EPT, WIDE_ITER><<<gw, s.T1, sw_bytes, st>>>(wa);
  }
  if ((e = cudaGetLastError()) != cudaSuccess) return LL_ERR_CUDA;
  if ((e = cudaMemcpyAsync(&hs, dst, sizeof(DevState), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return LL_ERR_CUDA;
  restore.enqueued = false;
  if (max_err) memcpy(max_err, &hs.err_bits, sizeof(float));
  if (hs.fault & 1u) return LL_ERR_TIMEOUT;
  // a word outside the exact FP64 range: the digits are not valid, and the
  // roundoff reading may not show it; report it as ll_step does, as the
  // largest possible error, so that the caller's roundoff policy fires
  if ((hs.fault & 2u) && max_err) *max_err = 1.0f;
  return LL_OK;
}

// ---------------------------------------------------------------------------
// Batched mode: many exponents of any lengths advance together.
//
// Every member is an ordinary context (own buffers, tables, stream and
// shape).  One step of K iterations for the whole batch is a single CUDA
// graph: each member's chain of K x (tall, wide) launches is its own branch,
// the branches fork from and join back to the batch stream, and the GPU runs
// the independent branches concurrently.  A member runs exactly the kernels it
// would run alone, so its residues are the solo residues.
// Members of one FFT length whose passes both have specialised kernels run
// as a length class: one launch per pass for all of them (blockIdx.x =
// member * units + unit), the members' kernel arguments in a device array.
struct BatchClass {
  std::vector<int> idx;  // members
  const StaticTall *st = nullptr;
  const StaticWide *sw = nullptr;
  TallArgs *d_ta = nullptr;
  WideArgs *d_wa = nullptr;
  int tall_units = 0, wide_units = 0, T1 = 0, T2 = 0;
  size_t smem_t = 0, smem_w = 0;
  bool pdl = false;
  cudaStream_t stream = nullptr;
};

struct ll_batch {
  int device = 0;
  std::vector<ll_ctx *> members;
  cudaStream_t stream = nullptr;
  std::vector<cudaEvent_t> events;  // [0] fork, [1..] joins
  int graph_iters = 0;
  bool by_class = true;                 // one launch per pass per length class (else per member)
  std::vector<BatchClass> classes;
  std::vector<int> singles;             // members launched on their own
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  std::string err;
};

static void free_batch(ll_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaEvent_t e : b->events) cudaEventDestroy(e);
  for (BatchClass &k : b->classes) {
    if (k.d_ta) cudaFree(k.d_ta);
    if (k.d_wa) cudaFree(k.d_wa);
    if (k.stream) cudaStreamDestroy(k.stream);
  }
  if (b->stream) cudaStreamDestroy(b->stream);
  for (ll_ctx *c : b->members) ll_destroy(c);
  delete b;
}

// Groups the members into length classes (the rest stay singles), uploads
// the classes' argument arrays and creates a stream per class.
static ll_status build_classes(ll_batch *b) {
  std::vector<int> order;
  for (size_t i = 0; i < b->members.size(); ++i) {
    const ll_ctx *c = b->members[i];
    if (!(c->shape.sw && c->shape.st && c->shape.st->batch)) {
      b->singles.push_back((int)i);
      continue;
    }
    BatchClass *k = nullptr;
    for (BatchClass &x : b->classes)
      if (b->members[(size_t)x.idx[0]]->n == c->n) k = &x;
    if (!k) {
      b->classes.emplace_back();
      k = &b->classes.back();
    }
    k->idx.push_back((int)i);
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  for (BatchClass &k : b->classes) {
    const ll_ctx *c0 = b->members[(size_t)k.idx[0]];
    const Shape &s = c0->shape;
    k.st = s.st;
    k.sw = s.sw;
    k.tall_units = tall_grid(s);
    k.wide_units = s.H / s.G;
    k.T1 = s.T1;
    k.T2 = s.T2;
    k.smem_t = shape_tall_smem(s);
    k.smem_w = shape_wide_smem(s);
    std::vector<TallArgs> ta;
    std::vector<WideArgs> wa;
    for (int i : k.idx) {
      ta.push_back(b->members[(size_t)i]->ta);
      wa.push_back(b->members[(size_t)i]->wa);
    }
    if (upload(&k.d_ta, ta) != cudaSuccess || upload(&k.d_wa, wa) != cudaSuccess ||
        cudaStreamCreateWithFlags(&k.stream, cudaStreamNonBlocking) != cudaSuccess)
      return LL_ERR_CUDA;
    // chained launches when both passes of the class run in a few waves
    int bw = 0, bt = 0;
    const long long m = (long long)k.idx.size();
    if (sms > 0 &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bw, k.sw->iter_batch, k.T1, k.smem_w) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, k.st->batch, k.T2, k.smem_t) == cudaSuccess && bw > 0 &&
        bt > 0) {
      const long long ww = (m * k.wide_units + (long long)sms * bw - 1) / ((long long)sms * bw);
      const long long wt = (m * k.tall_units + (long long)sms * bt - 1) / ((long long)sms * bt);
      k.pdl = ww <= 4 && wt <= 4;
    }
  }
  return LL_OK;
}

static void launch_class(const void *kern, const void *arr, int units, int count, int threads, size_t smem,
                         cudaStream_t st, bool chained) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(units * count));
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = chained ? 1 : 0;
  void *argv[] = {(void *)&arr, (void *)&units};
  cudaLaunchKernelExC(&cfg, kern, argv);
}

extern "C" {

ll_status ll_batch_create(int device, int32_t count, const uint32_t *q, const uint32_t *n, int32_t graph_iters,
                          ll_batch **out) {
  if (!out || count <= 0 || !q || !n) return LL_ERR_ARG;
  *out = nullptr;
  ll_batch *b = new ll_batch();
  b->device = device;
  b->graph_iters = graph_iters > 0 ? graph_iters : 10;
  ll_tuning t{};
  t.graph_iters = -1;  // members never capture their own graphs
  for (int32_t i = 0; i < count; ++i) {
    ll_ctx *c = nullptr;
    ll_status s = ll_create(device, q[i], n[i], &t, &c);
    if (s != LL_OK) {
      free_batch(b);
      return s;
    }
    b->members.push_back(c);
  }
  cudaSetDevice(device);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    free_batch(b);
    return LL_ERR_CUDA;
  }
  const ll_status cs = build_classes(b);
  if (cs != LL_OK) {
    free_batch(b);
    return cs;
  }
  b->events.resize((size_t)count + b->classes.size() + 1, nullptr);
  for (auto &e : b->events)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      free_batch(b);
      return LL_ERR_CUDA;
    }
  *out = b;
  return LL_OK;
}

void ll_batch_destroy(ll_batch *b) { free_batch(b); }

int32_t ll_batch_size(const ll_batch *b) { return b ? (int32_t)b->members.size() : 0; }

ll_ctx *ll_batch_member(ll_batch *b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->members.size()) return nullptr;
  return b->members[(size_t)i];
}

ll_status ll_batch_start(ll_batch *b, const uint32_t *offsets) {
  if (!b) return LL_ERR_ARG;
  for (size_t i = 0; i < b->members.size(); ++i) {
    ll_status s = ll_start(b->members[i], offsets ? offsets[i] : 0);
    if (s != LL_OK) return s;
  }
  return LL_OK;
}

ll_status ll_batch_step(ll_batch *b, uint32_t iters, uint32_t flags, float *max_err) {
  if (!b) return LL_ERR_ARG;
  for (ll_ctx *c : b->members)
    if (!c->started) return LL_ERR_STATE;
  if (cudaSetDevice(b->device) != cudaSuccess) return LL_ERR_CUDA;
  const bool report = (flags & LL_REPORT) != 0;
  const uint32_t K = (uint32_t)b->graph_iters;
  const uint32_t plain = iters - (report && iters ? 1u : 0u);
  uint32_t done = 0;
  if (plain >= K) {
    if (!b->graph_exec) {
      if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return LL_ERR_CUDA;
      cudaEventRecord(b->events[0], b->stream);
      size_t ev = 1;
      std::vector<int> alone;
      if (b->by_class) {
        for (BatchClass &k : b->classes) {
          cudaStreamWaitEvent(k.stream, b->events[0], 0);
          const int m = (int)k.idx.size();
          for (uint32_t it = 0; it < K; ++it) {
            launch_class((const void *)k.st->batch, k.d_ta, k.tall_units, m, k.T2, k.smem_t, k.stream, it > 0 && k.pdl);
            launch_class((const void *)k.sw->iter_batch, k.d_wa, k.wide_units, m, k.T1, k.smem_w, k.stream, k.pdl);
          }
          cudaEventRecord(b->events[ev], k.stream);
          cudaStreamWaitEvent(b->stream, b->events[ev++], 0);
        }
        alone = b->singles;
      } else {
        for (size_t i = 0; i < b->members.size(); ++i) alone.push_back((int)i);
      }
      for (int i : alone) {
        ll_ctx *c = b->members[(size_t)i];
        cudaStreamWaitEvent(c->stream, b->events[0], 0);
        const uint32_t off0 = c->offset;
        for (uint32_t k = 0; k < K; ++k) {
          launch_tall(c, k > 0);
          launch_wide(c, WIDE_ITER, true);
        }
        c->offset = off0;
        cudaEventRecord(b->events[ev], c->stream);
        cudaStreamWaitEvent(b->stream, b->events[ev++], 0);
      }
      cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph);
      if (e != cudaSuccess) {
        b->err = cudaGetErrorString(e);
        return LL_ERR_CUDA;
      }
      if (cudaGraphInstantiate(&b->graph_exec, b->graph, 0) != cudaSuccess) return LL_ERR_CUDA;
    }
    // the members' streams must have finished earlier work (e.g. ll_start)
    for (ll_ctx *c : b->members) {
      cudaEvent_t ev = b->events[0];
      cudaEventRecord(ev, c->stream);
      cudaStreamWaitEvent(b->stream, ev, 0);
    }
    while (plain - done >= K) {
      if (cudaGraphLaunch(b->graph_exec, b->stream) != cudaSuccess) return LL_ERR_CUDA;
      for (ll_ctx *c : b->members)
        for (uint32_t k = 0; k < K; ++k) c->offset = (uint32_t)((2ull * c->offset) % c->q);
      done += K;
    }
    // later per-member work is ordered after the graph
    cudaEventRecord(b->events[0], b->stream);
    for (ll_ctx *c : b->members) cudaStreamWaitEvent(c->stream, b->events[0], 0);
  }
  for (size_t i = 0; i < b->members.size(); ++i) {
    ll_ctx *c = b->members[i];
    float e = 0.f;
    const uint32_t rest = iters - done;
    if (rest || flags) {
      ll_status s = ll_step(c, rest, flags, &e);
      if (s != LL_OK) return s;
    } else if (iters) {
      c->digits_current = false;
    }
    if (max_err) max_err[i] = e;
  }
  return LL_OK;
}

void *ll_batch_stream(const ll_batch *b) { return b ? (void *)b->stream : nullptr; }

ll_status ll_batch_group_by_length(ll_batch *b, int32_t on) {
  if (!b) return LL_ERR_ARG;
  if (b->graph_exec) return LL_ERR_STATE;  // the step graph is captured on the first step
  b->by_class = on != 0;
  return LL_OK;
}

int32_t ll_batch_classes(const ll_batch *b) { return b ? (int32_t)b->classes.size() : 0; }

ll_status ll_batch_sync(ll_batch *b) {
  if (!b) return LL_ERR_ARG;
  cudaSetDevice(b->device);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return LL_ERR_CUDA;
  for (ll_ctx *c : b->members)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return LL_ERR_CUDA;
  return LL_OK;
}

ll_status ll_batch_res64(ll_batch *b, uint64_t *res64) {
  if (!b || !res64) return LL_ERR_ARG;
  for (size_t i = 0; i < b->members.size(); ++i) {
    ll_status s = ll_res64(b->members[i], &res64[i]);
    if (s != LL_OK) return s;
  }
  return LL_OK;
}

}  // extern "C"
