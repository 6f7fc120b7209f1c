// Device building blocks of the B200 IBDWT engine: complex FP64 helpers,
// register-resident DFT kernels of radix 2/3/4/5/7/8/16, and an in-place
// mixed-radix Stockham FFT over rows held in shared memory.
//
// The FFT replaces the cuFFT Z2Z calls of CUDALucas (CUDALucas.cu:1888,
// :1890).  Sign convention: SIGN = +1 computes sum_j x_j e^{+2 pi i jk/L}
// (cuFFT's CUFFT_INVERSE), SIGN = -1 the conjugate transform; both are
// unnormalised.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace llb {

struct FftPlan {
  int L;          // transform length
  int nst;        // number of stages
  int radix[10];  // radix of each stage (product == L)
};

// Shared-memory layout: element i of the concatenated rows lives at pad(i).
// One 16-byte pad word per 16 elements spreads the stride-R writes of the
// early Stockham stages over the banks.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded(int n) { return n + (n >> 4) + 1; }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 conjg(double2 a) { return make_double2(a.x, -a.y); }
// a * (SIGN * i)
template <int SIGN>
__device__ __forceinline__ double2 mul_si(double2 a) {
  return SIGN > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// cos/sin of 2*pi*k/R (computed in 80-bit precision, rounded once).
#define C16_1 0.9238795325112867
#define S16_1 0.3826834323650898
#define SQH 0.7071067811865476
#define S3_1 0.8660254037844386
#define C5_1 0.30901699437494745
#define S5_1 0.9510565162951535
#define C5_2 (-0.8090169943749475)
#define S5_2 0.5877852522924731
#define C7_1 0.6234898018587335
#define S7_1 0.7818314824680298
#define C7_2 (-0.2225209339563144)
#define S7_2 0.9749279121818236
#define C7_3 (-0.9009688679024191)
#define S7_3 0.4338837391175581

template <int SIGN>
__device__ __forceinline__ void dft2(double2 &a, double2 &b) {
  double2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int SIGN>
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3) {
  double2 s0 = cadd(a0, a2), d0 = csub(a0, a2);
  double2 s1 = cadd(a1, a3), d1 = mul_si<SIGN>(csub(a1, a3));
  a0 = cadd(s0, s1);
  a2 = csub(s0, s1);
  a1 = cadd(d0, d1);
  a3 = csub(d0, d1);
}

template <int SIGN>
__device__ __forceinline__ void dft3(double2 *v) {
  double2 t1 = cadd(v[1], v[2]);
  double2 t2 = make_double2(fma(-0.5, t1.x, v[0].x), fma(-0.5, t1.y, v[0].y));
  double2 t3 = mul_si<SIGN>(cscale(csub(v[1], v[2]), S3_1));
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <int SIGN>
__device__ __forceinline__ void dft5(double2 *v) {
  double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  double2 a0 = v[0];
  double2 c1 = make_double2(a0.x + C5_1 * t1.x + C5_2 * t2.x, a0.y + C5_1 * t1.y + C5_2 * t2.y);
  double2 c2 = make_double2(a0.x + C5_2 * t1.x + C5_1 * t2.x, a0.y + C5_2 * t1.y + C5_1 * t2.y);
  double2 s1 = mul_si<SIGN>(make_double2(S5_1 * t3.x + S5_2 * t4.x, S5_1 * t3.y + S5_2 * t4.y));
  double2 s2 = mul_si<SIGN>(make_double2(S5_2 * t3.x - S5_1 * t4.x, S5_2 * t3.y - S5_1 * t4.y));
  v[0] = cadd(a0, cadd(t1, t2));
  v[1] = cadd(c1, s1);
  v[4] = csub(c1, s1);
  v[2] = cadd(c2, s2);
  v[3] = csub(c2, s2);
}

template <int SIGN>
__device__ __forceinline__ void dft7(double2 *v) {
  double2 p1 = cadd(v[1], v[6]), m1 = csub(v[1], v[6]);
  double2 p2 = cadd(v[2], v[5]), m2 = csub(v[2], v[5]);
  double2 p3 = cadd(v[3], v[4]), m3 = csub(v[3], v[4]);
  double2 a0 = v[0];
  double2 c1 = make_double2(a0.x + C7_1 * p1.x + C7_2 * p2.x + C7_3 * p3.x,
                            a0.y + C7_1 * p1.y + C7_2 * p2.y + C7_3 * p3.y);
  double2 c2 = make_double2(a0.x + C7_2 * p1.x + C7_3 * p2.x + C7_1 * p3.x,
                            a0.y + C7_2 * p1.y + C7_3 * p2.y + C7_1 * p3.y);
  double2 c3 = make_double2(a0.x + C7_3 * p1.x + C7_1 * p2.x + C7_2 * p3.x,
                            a0.y + C7_3 * p1.y + C7_1 * p2.y + C7_2 * p3.y);
  // sin(2 pi k c / 7) for (k,c): k=1: s1,s2,s3; k=2: s2,-s3,-s1; k=3: s3,-s1,s2
  double2 s1 = mul_si<SIGN>(make_double2(S7_1 * m1.x + S7_2 * m2.x + S7_3 * m3.x,
                                         S7_1 * m1.y + S7_2 * m2.y + S7_3 * m3.y));
  double2 s2 = mul_si<SIGN>(make_double2(S7_2 * m1.x - S7_3 * m2.x - S7_1 * m3.x,
                                         S7_2 * m1.y - S7_3 * m2.y - S7_1 * m3.y));
  double2 s3 = mul_si<SIGN>(make_double2(S7_3 * m1.x - S7_1 * m2.x + S7_2 * m3.x,
                                         S7_3 * m1.y - S7_1 * m2.y + S7_2 * m3.y));
  v[0] = cadd(a0, cadd(p1, cadd(p2, p3)));
  v[1] = cadd(c1, s1);
  v[6] = csub(c1, s1);
  v[2] = cadd(c2, s2);
  v[5] = csub(c2, s2);
  v[3] = cadd(c3, s3);
  v[4] = csub(c3, s3);
}

// 8-point DFT as 2 x 4: even/odd DFT4 then one radix-2 layer with w8^k.
template <int SIGN>
__device__ __forceinline__ void dft8(double2 *v) {
  dft4<SIGN>(v[0], v[2], v[4], v[6]);
  dft4<SIGN>(v[1], v[3], v[5], v[7]);
  // odd outputs: O0=v1, O1=v3, O2=v5, O3=v7 -> multiply by w8^k
  double2 o1 = v[3], o2 = v[5], o3 = v[7];
  o1 = make_double2(SQH * (o1.x - SIGN * o1.y), SQH * (o1.y + SIGN * o1.x));   // (1 + s i)/sqrt2
  o2 = mul_si<SIGN>(o2);
  o3 = make_double2(SQH * (-o3.x - SIGN * o3.y), SQH * (-o3.y + SIGN * o3.x)); // (-1 + s i)/sqrt2
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// 16-point DFT as 4 x 4 with twiddles w16^(c2*k1).
template <int SIGN>
__device__ __forceinline__ void dft16(double2 *v) {
  // index c = 4*c1 + c2, output k = k1 + 4*k2
#pragma unroll
  for (int c2 = 0; c2 < 4; ++c2) dft4<SIGN>(v[c2], v[4 + c2], v[8 + c2], v[12 + c2]);
  // now v[4*k1 + c2] = Y[c2][k1]; apply w16^(c2*k1)
  const double2 w1 = make_double2(C16_1, SIGN * S16_1);
  const double2 w2 = make_double2(SQH, SIGN * SQH);
  const double2 w3 = make_double2(S16_1, SIGN * C16_1);
  v[4 + 1] = cmul(v[4 + 1], w1);
  v[4 + 2] = cmul(v[4 + 2], w2);
  v[4 + 3] = cmul(v[4 + 3], w3);
  v[8 + 1] = cmul(v[8 + 1], w2);
  v[8 + 2] = mul_si<SIGN>(v[8 + 2]);
  v[8 + 3] = cmul(v[8 + 3], make_double2(-SQH, SIGN * SQH));
  v[12 + 1] = cmul(v[12 + 1], w3);
  v[12 + 2] = cmul(v[12 + 2], make_double2(-SQH, SIGN * SQH));
  v[12 + 3] = cmul(v[12 + 3], make_double2(-C16_1, -SIGN * S16_1));
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<SIGN>(v[4 * k1 + 0], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // leaves X[k1 + 4*k2] in v[4*k1 + k2]; out_slot<16> maps the order
}

// Register slot that holds output r of dft<R> (dft16 leaves its outputs
// transposed; all other kernels leave them in natural order).
template <int R>
__device__ __forceinline__ constexpr int out_slot(int r) {
  return R == 16 ? 4 * (r & 3) + (r >> 2) : r;
}

template <int R, int SIGN>
__device__ __forceinline__ void dft(double2 *v) {
  if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
  else if constexpr (R == 3) dft3<SIGN>(v);
  else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 5) dft5<SIGN>(v);
  else if constexpr (R == 7) dft7<SIGN>(v);
  else if constexpr (R == 8) dft8<SIGN>(v);
  else if constexpr (R == 16) dft16<SIGN>(v);
}

// One Stockham stage over B rows of length L (concatenated, padded) held in
// shared memory, in place: every thread loads all its butterflies into
// registers, the block synchronises, then all results are stored.
// NB bounds the butterflies per thread: B*L <= NB*R*blockDim.x.
// tw[e] = e^{+2 pi i e / L}.
template <int R, int NB, int SIGN>
__device__ __forceinline__ void fft_stage(double2 *s, int L, int B, int row0, int ns,
                                          const double2 *__restrict__ tw) {
  const int m = L / R;
  const int total = B * m;
  const int T = blockDim.x;
  const int step = L / (ns * R);
  double2 v[NB][R];
  int ob[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int bf = threadIdx.x + b * T;
    ob[b] = -1;
    if (bf < total) {
      const int row = bf / m;
      const int j = bf - row * m;
      const int k = j % ns;
      const int rb = (row0 + row) * L;
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = s[pad(rb + j + r * m)];
      if (ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          double2 w = __ldg(&tw[r * k * step]);
          v[b][r] = SIGN > 0 ? cmul(v[b][r], w) : cmulc(v[b][r], w);
        }
      }
      dft<R, SIGN>(v[b]);
      ob[b] = rb + (j - k) * R + k;
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (ob[b] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) s[pad(ob[b] + r * ns)] = v[b][out_slot<R>(r)];
    }
  }
  __syncthreads();
}

// Full transform of B rows; natural order in, natural order out.
// Requires B*L <= EPT*blockDim.x.  The plan lists the radices grouped in the
// fixed order 16, 8, 4, 2, 3, 5, 7 (see make_plan); each group is its own
// loop so that the register allocation of one radix does not constrain the
// others.
template <int R, int EPT, int SIGN>
__device__ __forceinline__ void fft_group(double2 *s, const FftPlan &P, int B, int row0, int &st, int &ns,
                                          const double2 *__restrict__ tw) {
#pragma unroll 1
  while (st < P.nst && P.radix[st] == R) {
    fft_stage<R, (EPT + R - 1) / R, SIGN>(s, P.L, B, row0, ns, tw);
    ns *= R;
    ++st;
  }
}

template <int EPT, int SIGN>
__device__ __forceinline__ void fft_rows_b(double2 *s, const FftPlan &P, int B, int row0,
                                           const double2 *__restrict__ tw) {
  int ns = 1, st = 0;
  fft_group<16, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<8, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<4, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<2, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<3, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<5, EPT, SIGN>(s, P, B, row0, st, ns, tw);
  fft_group<7, EPT, SIGN>(s, P, B, row0, st, ns, tw);
}

}  // namespace llb
