// Compile-time specialised tall/wide passes for row lengths L = 16 * M * 16
// (radix list 16, M, 16) and L = 256 (16, 16).
//
// Same mathematics and data layout as the generic kernels in engine.cu, but
// the radix list of the row transform is a template parameter, so every
// index, stride and loop bound is a constant, and the first radix is 16:
//  * a row of L elements is handled by TR = L/16 threads;
//  * the inverse transform runs the radix list backwards, so its last stage
//    (radix 16) leaves element m1 = t + r*TR of the row in register r of
//    thread t -- exactly the inputs of the forward transform's first stage.
//    The wide pass therefore rounds, carries and reweights in registers
//    between the two transforms, with no shared-memory round trip;
//  * the tall pass loads its first stage straight from HBM and stores its
//    last stage straight to HBM (both coalesced along the column).
// Included from engine.cu inside namespace llb, after the shared helpers.

template <int... Rs>
struct RList {
  static constexpr int N = sizeof...(Rs);
  static constexpr int a[N] = {Rs...};
  static constexpr int L = (Rs * ... * 1);
};

// Composite DFT of radix P*Q in registers: DFT_P over c1 for every c2,
// twiddles w_R^(c2*k1), DFT_Q over c2 for every k1.  Output k1 + P*k2 is
// left in v[Q*k1 + k2].
template <int P, int Q, int SIGN>
__device__ __forceinline__ void dft_pq(double2 *v) {
  constexpr int R = P * Q;
#pragma unroll
  for (int c2 = 0; c2 < Q; ++c2) {
    double2 w[P];
#pragma unroll
    for (int c1 = 0; c1 < P; ++c1) w[c1] = v[Q * c1 + c2];
    dft<P, SIGN>(w);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      double2 y = w[out_slot<P>(k1)];
      if (c2 != 0 && k1 != 0) {
        double2 t = wconst<R>(c2 * k1);
        y = SIGN > 0 ? cmul(y, t) : cmulc(y, t);
      }
      v[Q * k1 + c2] = y;
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < P; ++k1) {
    double2 w[Q];
#pragma unroll
    for (int c2 = 0; c2 < Q; ++c2) w[c2] = v[Q * k1 + c2];
    dft<Q, SIGN>(w);
#pragma unroll
    for (int k2 = 0; k2 < Q; ++k2) v[Q * k1 + k2] = w[out_slot<Q>(k2)];
  }
}

template <int R>
struct Split {  // factor P*Q of a composite radix (P = 0: prime kernel)
  static constexpr int P = R == 6 ? 2 : R == 9 ? 3 : R == 10 ? 2 : R == 12 ? 4 : R == 14 ? 2 : R == 20 ? 4 : 0;
  static constexpr int Q = P ? R / P : 0;
};

template <int R, int SIGN>
__device__ __forceinline__ void sdft(double2 *v) {
  if constexpr (Split<R>::P) dft_pq<Split<R>::P, Split<R>::Q, SIGN>(v);
  else dft<R, SIGN>(v);
}

template <int R>
__device__ __forceinline__ constexpr int sslot(int r) {
  if constexpr (Split<R>::P) return Split<R>::Q * (r % Split<R>::P) + r / Split<R>::P;
  else return out_slot<R>(r);
}

// Stage twiddles live in one table per row length, in stage order: for
// every stage s with NS_s > 1 (radices of the list a[] applied in order,
// NS_s = a[0]*...*a[s-1]) the entries w_{NS_s*R_s}^(r*k) for k < NS_s,
// r = 1..R_s-1, row k contiguous with an odd row stride (R-1 rounded up to
// odd) so that consecutive k fall in distinct shared-memory bank groups.
// The lists used are palindromic, so the reversed (inverse) order has the
// same stages and uses the same table.
__host__ __device__ constexpr int tw_stride(int R) { return (R - 1) | 1; }

template <class P, int I>
__host__ __device__ constexpr int tw_offset() {
  int off = 0, ns = 1;
  for (int i = 0; i < I; ++i) {
    if (ns > 1) off += ns * tw_stride(P::a[i]);
    ns *= P::a[i];
  }
  return off;
}
template <class P>
__host__ __device__ constexpr int tw_size() { return tw_offset<P, P::N>(); }

template <class P>
__host__ __device__ constexpr bool palindromic() {
  for (int i = 0; i < P::N; ++i)
    if (P::a[i] != P::a[P::N - 1 - i]) return false;
  return true;
}

// Shared-memory rows: element x of row `row` lives in slot row*RS + pad(x).
// RS = L + L/16 for the tall pass (two columns, as one padded array); the
// wide pass adds up to 7 slots per row so that the G rows of a CTA start
// 8/G bank groups apart (its row-interleaved global loads and stores then
// hit distinct banks).
template <int L>
__host__ __device__ constexpr int col_slots() { return L + L / 16; }
template <int L, int G>
__host__ __device__ constexpr int row_slots() {
  return L + L / 16 + (G > 1 ? ((8 / G - (L + L / 16) % 8) % 8 + 8) % 8 : 0);
}

// Barriers of the kernel bodies: the whole CTA (__syncthreads), or the first
// n threads of the CTA (named barrier `id`), which lets a body run on a part
// of a larger CTA.
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct PartSync {
  int id, n;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
  }
};

// One Stockham stage of every row of the CTA, in place in shared memory.
// Thread t of a row handles butterflies t, t+TR, ... (a guard skips the
// tail when L/R is not a multiple of TR).  `tw` points at this stage's
// twiddle block (NS rows of R-1 entries) in shared memory.
template <int L, int RS, int R, int NS, int SIGN, int TR, class S = CtaSync>
__device__ __forceinline__ void sstage(double2 *s, const double2 *tw, int row, int t, S sync = S()) {
  const int rb = row * RS;
  constexpr int M = L / R;
  constexpr int NB = (M + TR - 1) / TR;
  // When TR is a multiple of NS, every butterfly j = t + b*TR of this thread
  // has the same twiddle row k = t mod NS: load it once (small radices only;
  // for larger ones the registers it holds cost more than the loads).
  constexpr bool kShared = NS > 1 && NB > 1 && TR % NS == 0 && R <= 8;
  double2 wk[kShared ? R - 1 : 1];
  if constexpr (kShared) {
#pragma unroll
    for (int r = 1; r < R; ++r) wk[r - 1] = tw[(int)((unsigned)t % NS) * tw_stride(R) + r - 1];
  }
  double2 v[NB][R];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * TR;
    if (M % TR == 0 || j < M) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = s[rb + pad(j + r * M)];
      if constexpr (NS > 1) {
        const int k = (int)((unsigned)j % NS);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const double2 w = kShared ? wk[r - 1] : tw[k * tw_stride(R) + r - 1];
          v[b][r] = SIGN > 0 ? cmul(v[b][r], w) : cmulc(v[b][r], w);
        }
      }
      sdft<R, SIGN>(v[b]);
    }
  }
  // with one butterfly per thread and NS == L/R a thread stores exactly the
  // slots it loaded: no barrier between the loads and the stores
  if constexpr (!(NB == 1 && NS == M)) sync();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * TR;
    if (M % TR == 0 || j < M) {
      const int k = (int)((unsigned)j % NS);
      const int ob = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[rb + pad(ob + r * NS)] = v[b][sslot<R>(r)];
    }
  }
  sync();
}

// forward stages [I, E) (radix a[I], NS = a[0]*...*a[I-1])
template <class P, int RS, int I, int E, int NS, int TR, class S = CtaSync>
__device__ __forceinline__ void fwd_stages(double2 *s, const double2 *tw, int row, int t, S sync = S()) {
  if constexpr (I < E) {
    constexpr int R = P::a[I];
    sstage<P::L, RS, R, NS, +1, TR>(s, tw + tw_offset<P, I>(), row, t, sync);
    fwd_stages<P, RS, I + 1, E, NS * R, TR>(s, tw, row, t, sync);
  }
}

// inverse stages [I, E) of the reversed list (radix a[N-1-I])
template <class P, int RS, int I, int E, int NS, int TR, class S = CtaSync>
__device__ __forceinline__ void inv_stages(double2 *s, const double2 *tw, int row, int t, S sync = S()) {
  static_assert(palindromic<P>(), "inverse stages reuse the forward twiddle table");
  if constexpr (I < E) {
    constexpr int R = P::a[P::N - 1 - I];
    sstage<P::L, RS, R, NS, -1, TR>(s, tw + tw_offset<P, I>(), row, t, sync);
    inv_stages<P, RS, I + 1, E, NS * R, TR>(s, tw, row, t, sync);
  }
}

// First stage (radix 16, no twiddle) from registers x[t + r*TR]: of the
// forward transform (SIGN +1), or of the inverse one (SIGN -1, the reversed
// list starts with the same radix 16).
template <int L, int RS, int TR, int SIGN = +1>
__device__ __forceinline__ void first_stage_from_regs(double2 *s, double2 *v, int row, int t) {
  dft<16, SIGN>(v);
#pragma unroll
  for (int r = 0; r < 16; ++r) s[row * RS + pad(t * 16 + r)] = v[out_slot<16>(r)];
}

// Last stage (radix 16, NS = L/16) into registers: leaves X[t + r*TR] in
// o[r].  tw is the stage's twiddle block (k = t, 15 entries per k); SIGN -1
// for the inverse transform, +1 for the forward one.
template <int L, int RS, int TR, int SIGN = -1>
__device__ __forceinline__ void last_stage_to_regs(const double2 *s, const double2 *tw, double2 *o, int row, int t) {
  double2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = s[row * RS + pad(t + r * TR)];
#pragma unroll
  for (int r = 1; r < 16; ++r) v[r] = SIGN > 0 ? cmul(v[r], tw[t * 15 + r - 1]) : cmulc(v[r], tw[t * 15 + r - 1]);
  dft<16, SIGN>(v);
#pragma unroll
  for (int r = 0; r < 16; ++r) o[r] = v[out_slot<16>(r)];
}

template <class P>
constexpr int tall_threads() { return 2 * (P::L / 16); }

// Blocks per SM to ask of the register allocator: about 128 registers per
// thread, which leaves room for two or more CTAs per SM.
constexpr int min_blocks(int threads) {
  return 65536 / (threads * 128) > 32 ? 32 : 65536 / (threads * 128) > 1 ? 65536 / (threads * 128) : 1;
}

// Shared memory of the tall pass beyond the two columns: stage twiddles,
// the column twiddle factors w_N^(k*TR*r) of both columns (2 x 16) and the
// pairing-loop factors w_H^(j*2*TR) (8 entries).
// 16-byte asynchronous global -> shared copy (no register staging).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// L2 prefetches: a contiguous range (bulk, 16-byte aligned, size a multiple
// of 16) or one line.  When the state is larger than L2, a CTA prefetches the
// data of the unit about one wave ahead while it computes, so that unit's
// loads hit L2 instead of HBM.
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
template <int L>
constexpr bool kPrefetchRows = L >= 2048;

// Programmatic dependent launch.  The passes are launched with programmatic
// stream serialization, so a kernel may become resident while the previous
// pass drains and run its prologue (tables, twiddles, ticket) early.
// griddep_wait() returns once the previous kernel in the stream has completed
// and its writes are visible; every read of the state array and of the device
// state comes after it.  griddep_release() lets the next kernel start
// launching; it is called only after griddep_wait(), so two launches of the
// same pass never overlap.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Pairing strategy of the tall pass: when every warp holds threads of one
// column only (TR a multiple of 32), each thread pairs its own bins with the
// mirror bins of its partner thread in the other column (half exchange);
// otherwise all bins go through shared memory and the pairs are split over
// the CTA by index.
template <class P>
__host__ __device__ constexpr bool tall_half_exchange() { return (P::L / 16) % 32 == 0; }

template <class P>
__host__ __device__ constexpr int tall_extra() {
  return tw_size<P>() + 32 + 8 + (tall_half_exchange<P>() ? 16 + 4 * (P::L / 16) : 0);
}

// Tall pass for columns of length H = P::L (radix list 16, M, 16 or 16, 16); two
// columns per CTA.
// The column twiddle w_N^(k1*m2) of element m2 = t + r*TR is formed as
// w_N^(k1*t) (one table product per thread) times w_N^(k1*TR*r) (shared by
// the CTA), so no per-element table gathers are needed.
// The forward transform's last stage leaves bins t + r*TR (r < 16) of the
// thread's column in its registers and in its own shared-memory slots; the
// inverse transform's first stage reads exactly those slots.  Bin t + r*TR
// of column kA pairs with bin H-1-(t + r*TR) = (TR-1-t) + (15-r)*TR of
// column kB, which belongs to thread TR-1-t of the other column.  With the
// half exchange each thread computes the pairs of its bins r < 8 (the
// mirror bins, r >= 8 of the partner, come through shared memory) and writes
// the partner's results back into the partner's slots.  (CTA 0 holds the
// self-paired columns 0 and W/2 and always pairs through shared memory.)
template <class P, class S = CtaSync>
__device__ __forceinline__ void tall_body(const TallArgs &a, int blk, S sync = S()) {
  constexpr int H = P::L, TR = H / 16, T = 2 * TR, CS = col_slots<H>();
  constexpr bool kHalf = tall_half_exchange<P>();
  static_assert((P::N == 2 || P::N == 3) && P::a[0] == 16 && P::a[P::N - 1] == 16, "radix list 16, (M,) 16");
  extern __shared__ double2 sm[];
  double2 *stw = sm + padded(2 * H);
  double2 *wr = stw + tw_size<P>();  // w_N^(k*TR*r), both columns
  double2 *pj = wr + 32;             // w_H^(j*T), pairing by index
  double2 *fr = pj + 8;              // w_H^(r*TR), half exchange
  double2 *sbase = fr + 16;          // per thread: w_N^(k1*t), half exchange
  double2 *spair = sbase + T;        // per thread: w_N^kA * w_H^tA, half exchange
  const int c = blk;
  const int W = a.W;
  const bool special = (c == 0);
  const int kA = special ? 0 : c;
  const int kB = special ? W / 2 : W - c;
  const int col = threadIdx.x / TR, t = threadIdx.x - col * TR;
  const int k1 = col ? kB : kA;
  for (int i = threadIdx.x; i < tw_size<P>(); i += T) cp_async16(&stw[i], &a.stw[i]);
  for (int i = threadIdx.x; i < (kHalf ? 56 : 40); i += T) {  // one pass when T >= 56
    if (i < 32) {
      const int kk = i < 16 ? kA : kB, r = i & 15;
      wr[i] = omegaN(a.thi, a.tlo, a.ts, a.tmask, kk * TR * r);
    } else if (i < 40) {
      pj[i - 32] = __ldg(&a.twH[(i - 32) * T]);
    } else {
      fr[i - 40] = __ldg(&a.twH[(i - 40) * TR]);
    }
  }
  // with the half exchange the per-thread twiddle bases are parked in the
  // thread's own shared-memory slot while the transforms hold the registers
  // (tA is the column-kA bin row of the thread's pairs)
  double2 base = omegaN(a.thi, a.tlo, a.ts, a.tmask, k1 * t);
  if constexpr (kHalf) {
    sbase[threadIdx.x] = base;
    spair[threadIdx.x] = cmul(omegaN(a.thi, a.tlo, a.ts, a.tmask, kA), __ldg(&a.twH[col ? TR - 1 - t : t]));
  }
  griddep_wait();
  griddep_release();
  if (c == 0 && threadIdx.x == 0) {
    const uint32_t o = a.st->offset;  // CUDALucas.cu:1882, once per iteration
    a.st->offset = (uint32_t)((2ull * o) % a.q);
  }
  const double2 *src = a.A + (size_t)k1 * H;
  {
    double2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = src[t + r * TR];
    cp_async_wait_all();
    sync();
    if constexpr (kHalf) base = sbase[threadIdx.x];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = cmul(v[r], cmul(base, wr[col * 16 + r]));
    first_stage_from_regs<H, CS, TR>(sm, v, col, t);
  }
  if (kPrefetchRows<H> && a.pf && threadIdx.x == 0 && c + a.pf < W / 2) {
    const int c2 = c + a.pf;  // never 0: the pair of columns c2 and W - c2
    prefetch_l2_bulk(a.A + (size_t)c2 * H, H * (uint32_t)sizeof(double2));
    prefetch_l2_bulk(a.A + (size_t)(W - c2) * H, H * (uint32_t)sizeof(double2));
  }
  sync();
  fwd_stages<P, CS, 1, P::N - 1, 16, TR>(sm, stw, col, t, sync);
  double2 o[16];
  last_stage_to_regs<H, CS, TR, +1>(sm, stw + tw_offset<P, P::N - 1>(), o, col, t);
  double2 *own = sm + col * CS;  // own bin r: own[pad(t + r*TR)]
  if (kHalf && !special) {
#pragma unroll
    for (int r = 8; r < 16; ++r) own[pad(t + r * TR)] = o[r];
    sync();
    double2 *mir = sm + (col ^ 1) * CS;  // partner's bin 15-r: mir[pad(TR-1-t + (15-r)*TR)]
    // Swapping the two bins and conjugating w swaps the two results of
    // pair_square, so both columns make the same call: column kB passes its
    // own bin first and conj(w).
    const double2 wb = spair[threadIdx.x];
    const double sg = col ? -1.0 : 1.0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int ps = pad(TR - 1 - t + (15 - r) * TR);
      double2 zm = mir[ps];
      double2 w = cmul(wb, fr[col ? 15 - r : r]);
      w.y *= sg;
      pair_square(o[r], zm, w);
      mir[ps] = zm;
    }
    sync();
#pragma unroll
    for (int r = 8; r < 16; ++r) o[r] = own[pad(t + r * TR)];
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) own[pad(t + r * TR)] = o[r];
    sync();
    // pairing by index: i = threadIdx.x + j*T, w_H^i = w_H^threadIdx.x * pj[j]
    const double2 wt = __ldg(&a.twH[threadIdx.x]);
    if (!special) {
      const double2 wb = cmul(omegaN(a.thi, a.tlo, a.ts, a.tmask, kA), wt);
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // bin k2 of column kA <-> bin H-1-k2 of column kB
        const int k2 = threadIdx.x + j * T;
        double2 za = sm[pad(k2)], zb = sm[pad(2 * H - 1 - k2)];
        pair_square(za, zb, cmul(wb, pj[j]));
        sm[pad(k2)] = za;
        sm[pad(2 * H - 1 - k2)] = zb;
      }
    } else {
      const int half = H / 2;
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // column 0: k2 <-> (H-k2) mod H, w_N^(W*k2) = w_H^k2
        const int i = threadIdx.x + j * T;
        if (i <= half) {
          const int p = (H - i) % H;
          double2 za = sm[pad(i)], zb = sm[pad(p)];
          pair_square(za, zb, cmul(wt, pj[j]));
          sm[pad(i)] = za;
          if (p != i) sm[pad(p)] = zb;
        }
      }
      const double2 wb = cmul(omegaN(a.thi, a.tlo, a.ts, a.tmask, W / 2), wt);
#pragma unroll
      for (int j = 0; j < 8; ++j) {  // column W/2: k2 <-> H-1-k2
        const int i = threadIdx.x + j * T;
        if (i < half) {
          double2 za = sm[pad(H + i)], zb = sm[pad(2 * H - 1 - i)];
          pair_square(za, zb, cmul(wb, pj[j]));
          sm[pad(H + i)] = za;
          sm[pad(2 * H - 1 - i)] = zb;
        }
      }
    }
    sync();
#pragma unroll
    for (int r = 0; r < 16; ++r) o[r] = own[pad(t + r * TR)];
  }
  sync();  // every thread's slot reads are done before the stage-0 stores
  first_stage_from_regs<H, CS, TR, -1>(sm, o, col, t);
  sync();
  inv_stages<P, CS, 1, P::N - 1, 16, TR>(sm, stw, col, t, sync);
  last_stage_to_regs<H, CS, TR>(sm, stw + tw_offset<P, P::N - 1>(), o, col, t);
  double2 *dst = a.A + (size_t)k1 * H;
  if constexpr (kHalf) base = sbase[threadIdx.x];
#pragma unroll
  for (int r = 0; r < 16; ++r) dst[t + r * TR] = cmulc(o[r], cmul(base, wr[col * 16 + r]));
}

template <class P>
__global__ void __launch_bounds__(tall_threads<P>(), min_blocks(tall_threads<P>())) tall_static(TallArgs a) {
  tall_body<P>(a, blockIdx.x);
}

// All stages of the radix list P in list order, in shared memory (Stockham:
// natural order in and out); SIGN -1 with conjugate twiddles is the inverse
// transform over the same twiddle table.
template <class P, int RS, int I, int NS, int TR, int SIGN, class S = CtaSync>
__device__ __forceinline__ void all_stages(double2 *s, const double2 *tw, int row, int t, S sync = S()) {
  if constexpr (I < P::N) {
    constexpr int R = P::a[I];
    sstage<P::L, RS, R, NS, SIGN, TR>(s, tw + tw_offset<P, I>(), row, t, sync);
    all_stages<P, RS, I + 1, NS * R, TR, SIGN>(s, tw, row, t, sync);
  }
}

// One Stockham stage of one row with TR threads, like sstage, but the
// elements are read through ld(e, j, r) and the outputs written through
// st(e, j, r, v): e is the index within the row, j the butterfly and r the
// element of the butterfly (loads: e = j + r*L/R; stores of the last stage,
// where NS = L/R: e = j + r*NS).  INPLACE: the stage reads and writes the same
// slots, so a barrier separates the loads from the stores.
template <int L, int R, int NS, int SIGN, int TR, bool INPLACE, class S, class LD, class ST>
__device__ __forceinline__ void fstage(const double2 *tw, int t, S sync, LD ld, ST st) {
  constexpr int M = L / R;
  constexpr int NB = (M + TR - 1) / TR;
  constexpr bool kShared = NS > 1 && NB > 1 && TR % NS == 0 && R <= 8;
  double2 wk[kShared ? R - 1 : 1];
  if constexpr (kShared) {
#pragma unroll
    for (int r = 1; r < R; ++r) wk[r - 1] = tw[(int)((unsigned)t % NS) * tw_stride(R) + r - 1];
  }
  double2 v[NB][R];
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * TR;
    if (M % TR == 0 || j < M) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = ld(j + r * M, j, r);
      if constexpr (NS > 1) {
        const int k = (int)((unsigned)j % NS);
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const double2 w = kShared ? wk[r - 1] : tw[k * tw_stride(R) + r - 1];
          v[b][r] = SIGN > 0 ? cmul(v[b][r], w) : cmulc(v[b][r], w);
        }
      }
      sdft<R, SIGN>(v[b]);
    }
  }
  if constexpr (INPLACE && !(NB == 1 && NS == M)) sync();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * TR;
    if (M % TR == 0 || j < M) {
      const int k = (int)((unsigned)j % NS);
      const int ob = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) st(ob + r * NS, j, r, v[b][sslot<R>(r)]);
    }
  }
  sync();
}

// All stages of the radix list P: the first reads through ld0, the last
// writes through stN (both in place when they are the plain ld/st), the
// others read and write the row in place through ld/st.
// FIRSTIN: the first stage's loads read the row (or must be ordered before
// its stores into the row, e.g. reads of other slots by other threads): a
// barrier between its loads and stores.  LASTIN: the last stage stores into
// the row it reads; otherwise it stores elsewhere (global memory, another
// CTA, registers) and its closing barrier still orders its loads before
// later writes to the row.
template <class P, int I, int NS, int TR, int SIGN, bool FIRSTIN, bool LASTIN, class S, class LD0, class STN, class LD,
          class ST>
__device__ __forceinline__ void fall_stages(const double2 *tw, int t, S sync, LD0 ld0, STN stN, LD ld, ST st) {
  static_assert(P::N >= 2, "first and last stage distinct");
  if constexpr (I < P::N) {
    constexpr int R = P::a[I];
    const double2 *tws = tw + tw_offset<P, I>();
    if constexpr (I == 0) fstage<P::L, R, NS, SIGN, TR, FIRSTIN>(tws, t, sync, ld0, st);
    else if constexpr (I == P::N - 1) fstage<P::L, R, NS, SIGN, TR, LASTIN>(tws, t, sync, ld, stN);
    else fstage<P::L, R, NS, SIGN, TR, true>(tws, t, sync, ld, st);
    fall_stages<P, I + 1, NS * R, TR, SIGN, FIRSTIN, LASTIN>(tw, t, sync, ld0, stN, ld, st);
  }
}

// Tall pass for column lengths H = P::L outside the 16 x M x 16 family (any
// radix list of 2..16): PP column pairs per CTA, TC threads per column, every
// stage in shared memory.  A column is loaded with the twiddle w_N^(k1*m2)
// applied, transformed, paired by index with its mirror column (bins k2 and
// H-1-k2; pair 0 holds the self-paired columns 0 and W/2), transformed back
// with conjugate twiddles and stored with the conjugate twiddle.  The same
// arithmetic as the generic tall kernel, with every index and loop bound a
// constant.
// Shared memory of a tall_any CTA (double2 entries): 2*PP padded columns,
// the stage twiddles, and per column the factors w_N^(k1*M0*r) of the first
// stage's loads (r < a[0], M0 = H/a[0]) and w_N^(k1*NS*r) of the last
// stage's stores (r < a[N-1], NS = H/a[N-1]).
template <class P, int PP>
__host__ __device__ constexpr int tall_any_smem() {
  return 2 * PP * col_slots<P::L>() + tw_size<P>() + 2 * PP * (P::a[0] + P::a[P::N - 1]);
}

template <class P, int TC, int PP, class S = CtaSync>
__device__ __forceinline__ void tall_any_body(const TallArgs &a, int blk, S sync = S()) {
  constexpr int H = P::L, CS = col_slots<H>(), T = 2 * PP * TC;
  constexpr int R0 = P::a[0], RN = P::a[P::N - 1], M0 = H / R0, NSN = H / RN, FS = R0 + RN;
  extern __shared__ double2 sm[];
  double2 *stw = sm + 2 * PP * CS;
  double2 *fac = stw + tw_size<P>();
  const int units = a.W / 2;
  const int col = threadIdx.x / TC, t = threadIdx.x - col * TC;  // col < 2*PP
  const int pl = col >> 1;
  const int c = blk * PP + pl;  // column pair
  const bool active = c < units;
  const bool special = c == 0;
  const int W = a.W;
  const int kA = special ? 0 : c, kB = special ? W / 2 : W - c;
  // column of this thread (column 0 for the threads of a pair past the last
  // one: they read valid memory and store nothing)
  const int k1 = !active ? 0 : (col & 1) ? kB : kA;
  for (int i = threadIdx.x; i < tw_size<P>(); i += T) cp_async16(&stw[i], &a.stw[i]);
  for (int i = threadIdx.x; i < 2 * PP * FS; i += T) {
    const int cc = i / FS, r = i - cc * FS;
    const int cp = blk * PP + (cc >> 1);
    const int kk = cp >= units ? 0 : (cc & 1) ? (cp == 0 ? W / 2 : W - cp) : cp;
    fac[i] = omegaN(a.thi, a.tlo, a.ts, a.tmask, r < R0 ? kk * M0 * r : kk * NSN * (r - R0));
  }
  griddep_wait();
  griddep_release();
  if (blk == 0 && threadIdx.x == 0) {
    const uint32_t o = a.st->offset;  // CUDALucas.cu:1882, once per iteration
    a.st->offset = (uint32_t)((2ull * o) % a.q);
  }
  double2 *row = sm + col * CS;
  const double2 *fc = fac + col * FS;
  double2 *gcol = a.A + (size_t)k1 * H;
  cp_async_wait_all();
  sync();
  // the column twiddle w_N^(k1*m2) of element m2 = j + r*X (a butterfly j of
  // the first or last stage) is w_N^(k1*j) (once per butterfly) times the
  // stage's factor r of this column
  double2 base = make_double2(1.0, 0.0);
  auto ld = [&](int e, int, int) { return row[pad(e)]; };
  auto st = [&](int e, int, int, double2 v) { row[pad(e)] = v; };
  auto ld_first = [&](int e, int j, int r) {
    if (r == 0) base = omegaN(a.thi, a.tlo, a.ts, a.tmask, k1 * j);
    return active ? cmul(gcol[e], r == 0 ? base : cmul(base, fc[r])) : make_double2(0.0, 0.0);
  };
  fall_stages<P, 0, 1, TC, +1, false, true>(stw, t, sync, ld_first, st, ld, st);
  if (active) {
    const int ti = threadIdx.x - 2 * pl * TC;  // thread of the pair, < 2*TC
    double2 *ra = sm + 2 * pl * CS, *rb = ra + CS;
    // pairing twiddle w_N^(kb + W*k2) = w_N^kb * w_H^k2
    if (!special) {
      const double2 wb = omegaN(a.thi, a.tlo, a.ts, a.tmask, kA);
      for (int k2 = ti; k2 < H; k2 += 2 * TC) {  // bin k2 of column kA <-> bin H-1-k2 of column kB
        double2 za = ra[pad(k2)], zb = rb[pad(H - 1 - k2)];
        pair_square(za, zb, cmul(wb, __ldg(&a.twH[k2])));
        ra[pad(k2)] = za;
        rb[pad(H - 1 - k2)] = zb;
      }
    } else {
      for (int i = ti; i <= H / 2; i += 2 * TC) {  // column 0: k2 <-> (H-k2) mod H
        const int p2 = (H - i) % H;
        double2 za = ra[pad(i)], zb = ra[pad(p2)];
        pair_square(za, zb, __ldg(&a.twH[i]));
        ra[pad(i)] = za;
        if (p2 != i) ra[pad(p2)] = zb;
      }
      const double2 wb = omegaN(a.thi, a.tlo, a.ts, a.tmask, W / 2);
      for (int i = ti; i < H / 2; i += 2 * TC) {  // column W/2: k2 <-> H-1-k2
        double2 za = rb[pad(i)], zb = rb[pad(H - 1 - i)];
        pair_square(za, zb, cmul(wb, __ldg(&a.twH[i])));
        rb[pad(i)] = za;
        rb[pad(H - 1 - i)] = zb;
      }
    }
  }
  sync();
  auto st_last = [&](int e, int j, int r, double2 v) {
    if (r == 0) base = omegaN(a.thi, a.tlo, a.ts, a.tmask, k1 * j);
    if (active) gcol[e] = cmulc(v, r == 0 ? base : cmul(base, fc[R0 + r]));
  };
  fall_stages<P, 0, 1, TC, -1, true, false>(stw, t, sync, ld, st_last, ld, st);
}

template <class P, int TC, int PP>
__global__ void __launch_bounds__(2 * PP * TC, min_blocks(2 * PP * TC)) tall_any(TallArgs a) {
  tall_any_body<P, TC, PP>(a, blockIdx.x);
}

template <class P, int G>
__host__ __device__ constexpr int wide_threads() { return G * (P::L / 16); }

// Nearest integer of x for |x| < 2^51 (ties to even) by adding and removing
// 1.5*2^52: two FP64 adds instead of a rounding instruction.  The _rn
// intrinsics are never contracted or reassociated.  The carry splits below
// apply it to values below 2^37 in magnitude.
__device__ __forceinline__ double rnd_int(double x) {
  return __dsub_rn(__dadd_rn(x, 6755399441055744.0), 6755399441055744.0);
}

// Wide pass for rows of length W = P::L; G rows per CTA.
// The carry arithmetic runs in FP64 on integer-valued doubles (all values
// stay below 2^53 and every scaling is by a power of two, so every step is
// exact); carries are handed over as doubles, through shared memory between
// the rows of a CTA and through global memory from CTA to CTA.
// blk: the CTA's row group for WIDE_INIT (the iteration modes take tickets)
template <class P, int G, int MODE, bool BATCH, class S = CtaSync>
__device__ __forceinline__ void wide_body(const WideArgs &a, int blk, S sync = S()) {
  constexpr int W = P::L, TR = W / 16, T = G * TR;
  static_assert(P::a[0] == 16, "first radix must be 16");
  extern __shared__ double2 sm[];
  constexpr int RS = row_slots<W, G>();
  double2 *stw = sm + G * RS;
  __shared__ int s_g;
  __shared__ float s_err[32];
  __shared__ uint32_t s_fault;
  if (threadIdx.x == 0) {
    s_fault = 0;
    s_g = MODE == WIDE_INIT ? (BATCH ? blk : (int)blockIdx.x)
                            : (int)(atomicAdd(&a.st->ticket, 1ull) % (unsigned long long)a.ngroups);
  }
  for (int i = threadIdx.x; i < tw_size<P>(); i += T) cp_async16(&stw[i], &a.stw[i]);
  sync();
  const int g = s_g;
  const int H = a.H;
  const int m2b = g * G;
  // The G rows of an element column m1 sit in adjacent lanes.  With G >= 2
  // the global loads and stores of A[m1*H + m2b + row] then cover whole
  // 32-byte sectors, so the edge stages of the row transforms read and write
  // global memory directly; a single row (G = 1) touches half sectors, and
  // is staged through shared memory with cp.async instead.
  constexpr bool kDirect = G > 1;
  const int row = threadIdx.x % G, t = threadIdx.x / G;
  const int m2 = m2b + row;
  const int n = (int)a.n, bb = (int)a.b, qn = (int)a.qn;
  // Word s (0, 1) of element (m1 = t + r*TR, m2) has weight exponent
  // e = (E_s - colD[r]) mod n with the per-thread E_s = rowE + colF[t] mod n,
  // so its weight is Wt_s * colS[r] (or * colS2[r] when E_s < colD[r]).
  int E0 = __ldg(&a.rowE[2 * m2]) + __ldg(&a.colF[t]);
  int E1 = __ldg(&a.rowE[2 * m2 + 1]) + __ldg(&a.colF[t]);
  const double cwt = __ldg(&a.colW[t]);
  const double W0 = __ldg(&a.rowW[2 * m2]) * cwt * (E0 >= n ? 0.5 : 1.0);
  const double W1 = __ldg(&a.rowW[2 * m2 + 1]) * cwt * (E1 >= n ? 0.5 : 1.0);
  if (E0 >= n) E0 -= n;
  if (E1 >= n) E1 -= n;
  const double p2lo = (double)(1 << qn), p2hi = 2.0 * p2lo;
  const double ip2lo = 1.0 / p2lo, ip2hi = 0.5 * ip2lo;
  double2 x[16];
  double emax = 0.0;
  bool out_of_range = false;
  double Wi0 = 0.0, Wi1 = 0.0;
  if (MODE != WIDE_INIT) {
    const double cwit = __ldg(&a.colWi[t]);
    Wi0 = __ldg(&a.rowWi[2 * m2]) * cwit * (__ldg(&a.rowE[2 * m2]) + __ldg(&a.colF[t]) >= n ? 2.0 : 1.0);
    Wi1 = __ldg(&a.rowWi[2 * m2 + 1]) * cwit * (__ldg(&a.rowE[2 * m2 + 1]) + __ldg(&a.colF[t]) >= n ? 2.0 : 1.0);
  }
  // everything above reads constant tables only; the state array, the
  // digits and the device state are read after the previous pass completed
  griddep_wait();
  griddep_release();
  if (MODE != WIDE_INIT) {
    if constexpr (kDirect) {
      // the inverse transform's first stage (radix 16, no twiddle) works on
      // elements t + r*TR of the row: straight from global memory
      double2 v[16];
      const double2 *src = a.A + m2;
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = src[(size_t)(t + r * TR) * H];
      first_stage_from_regs<W, RS, TR, -1>(sm, v, row, t);
    } else {
      for (int k1 = threadIdx.x; k1 < W; k1 += T) cp_async16(&sm[pad(k1)], &a.A[(size_t)k1 * H + m2b]);
    }
    // (compiled for long rows only: only states larger than L2 prefetch, and
    // those have rows of 2048 and more)
    if (kPrefetchRows<W> && a.pf && g + a.pf < a.ngroups) {
      const double2 *nxt = a.A + (size_t)(g + a.pf) * G + row;
#pragma unroll
      for (int r = 0; r < 16; ++r) prefetch_l2(nxt + (size_t)(t + r * TR) * H);
    }
    // the -2 (bit (offset+1) mod q, CUDALucas.cu:1882-1886) hits at most one
    // word; locate it once: element register r_sub, word w_sub
    const uint32_t off = a.st->offset;
    const uint32_t pos = (off + 1) % a.q;
    const uint32_t dw = (uint32_t)(((unsigned long long)pos * a.n) / a.q);
    const uint32_t sdw = (uint32_t)(((unsigned long long)dw * a.q + a.n - 1) / a.n);
    const double sub = (double)(1u << (pos - sdw));
    int r_sub = -1;
    {
      const uint32_t me = dw >> 1, mm1 = me / (uint32_t)H, mm2 = me - mm1 * (uint32_t)H;
      if ((int)mm2 == m2 && (int)(mm1 % TR) == t) r_sub = (int)(mm1 / TR);
    }
    const bool w_sub = dw & 1;
    cp_async_wait_all();
    sync();
    if constexpr (kDirect) inv_stages<P, RS, 1, P::N - 1, 16, TR>(sm, stw, row, t, sync);
    else inv_stages<P, RS, 0, P::N - 1, 1, TR>(sm, stw, row, t, sync);
    double2 u[16];
    last_stage_to_regs<W, RS, TR>(sm, stw + tw_offset<P, P::N - 1>(), u, row, t);
    sync();  // shared memory is reused for the carry hand-off below

    // Carry in FP64 only (no integer conversions).  Phase 1 leaves, in the
    // shared-memory slot of element (row, m1), the packed pair
    // l0 + d1p*2^24 (|l0|, |d1p| <= 2^(bits-1) < 2^23, so the pair is exact
    // and separable) and the element's outgoing carry.
    double2 *ks = sm + row * RS + t;  // ks[r*TR]: element m1 = t + r*TR
    double *gcd = reinterpret_cast<double *>(a.carry);
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m1 = t + r * TR;
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const int e0 = E0 - D + (n0 ? n : 0), e1 = E1 - D + (n1 ? n : 0);
      const double t0 = u[r].x * (Wi0 * (n0 ? a.colSi2[r] : a.colSi[r]));
      const double t1 = u[r].y * (Wi1 * (n1 ? a.colSi2[r] : a.colSi[r]));
      double r0 = rint(t0), r1 = rint(t1);
      emax = fmax(emax, fmax(fabs(t0 - r0), fabs(t1 - r1)));
      // at 2^51 and above (or NaN) a double has no fraction bits left for the
      // roundoff reading, and the exact carry split below no longer holds
      if (!(fabs(t0) < 0x1p51 && fabs(t1) < 0x1p51)) out_of_range = true;
      if (r == r_sub) {
        if (w_sub) r1 -= sub;
        else r0 -= sub;
      }
      const bool big0 = e0 < bb, big1 = e1 < bb;
      const double P0 = big0 ? p2hi : p2lo, I0 = big0 ? ip2hi : ip2lo;
      const double P1 = big1 ? p2hi : p2lo, I1 = big1 ? ip2hi : ip2lo;
      // balanced splits r = h*2^bits + l; word 1 takes high_0 and is
      // balanced again; the outgoing carry high_1 + (carry of that balance)
      // depends on this element's own words only
      const double h0 = rnd_int(r0 * I0), l0 = fma(-h0, P0, r0);
      const double h1 = rnd_int(r1 * I1), l1 = fma(-h1, P1, r1);
      const double tt1 = l1 + h0;
      const double k1c = rnd_int(tt1 * I1);
      const double d1p = fma(-k1c, P1, tt1);
      const double co = h1 + k1c;
      ks[r * TR] = make_double2(fma(d1p, 0x1p24, l0), co);
      if (row == G - 1) gcd[(size_t)g * W + m1] = co;
    }
    // Hand-off warp by warp: warp w holds the same element columns m1 in
    // every CTA, so it publishes its last row's carries with its own flag
    // and waits only for the flag of warp w of the predecessor.  __syncwarp
    // orders the lanes' stores and loads around lane 0's release store and
    // acquire load.  (The wrap into CTA 0 shifts m1 by one across warps, so
    // CTA 0 waits for all warps of the last CTA.)
    const int pred = g == 0 ? a.ngroups - 1 : g - 1;
    constexpr int NW = T / 32;
    static_assert(T % 32 == 0 && NW <= kWarpFlags, "whole warps, one flag each");
    const int warp = threadIdx.x >> 5;
    __syncwarp();
    if ((threadIdx.x & 31) == 0)
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&a.flags[g * kWarpFlags + warp]), "r"(1u) : "memory");
    if (g != 0) {
      if ((threadIdx.x & 31) == 0) {
        uint32_t *f = &a.flags[pred * kWarpFlags + warp];
        if (!wait_flag(f)) atomicOr(&s_fault, 1u);
        *f = 0;
      }
      __syncwarp();
    } else {
      sync();
      if (threadIdx.x == 0) {
        for (int w = 0; w < NW; ++w) {
          uint32_t *f = &a.flags[pred * kWarpFlags + w];
          if (!wait_flag(f)) s_fault |= 1u;
          *f = 0;
        }
      }
      sync();
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m1 = t + r * TR;
      const double cin = row > 0 ? sm[(row - 1) * RS + m1].y
                                 : __ldcg(&gcd[(size_t)pred * W + (g == 0 ? (m1 == 0 ? W - 1 : m1 - 1) : m1)]);
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const int e0 = E0 - D + (n0 ? n : 0);
      const bool big0 = e0 < bb;
      const double P0 = big0 ? p2hi : p2lo, I0 = big0 ? ip2hi : ip2lo;
      const double pk = ks[r * TR].x;
      const double d1p = rnd_int(pk * 0x1p-24), l0 = fma(-d1p, 0x1p24, pk);
      const double tt0 = l0 + cin;
      const double k0 = rnd_int(tt0 * I0);
      const double d0 = fma(-k0, P0, tt0);
      const double d1 = d1p + k0;
      if (MODE == WIDE_REPORT) {
        const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
        a.xint[j0] = (int32_t)d0;
        a.xint[j0 + 1] = (int32_t)d1;
      }
      x[r] = make_double2(d0 * (W0 * (n0 ? a.colS2[r] : a.colS[r])), d1 * (W1 * (n1 ? a.colS2[r] : a.colS[r])));
    }
    sync();  // carry reads done before the data region is rewritten
  } else {
    cp_async_wait_all();
    sync();
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int m1 = t + r * TR;
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
      x[r] = make_double2((double)a.xint[j0] * (W0 * (n0 ? a.colS2[r] : a.colS[r])),
                          (double)a.xint[j0 + 1] * (W1 * (n1 ? a.colS2[r] : a.colS[r])));
    }
  }
  first_stage_from_regs<W, RS, TR>(sm, x, row, t);
  sync();
  if constexpr (kDirect) {
    fwd_stages<P, RS, 1, P::N - 1, 16, TR>(sm, stw, row, t, sync);
    // the last stage (radix 16) leaves elements t + r*TR in registers: store
    // them straight to global memory
    last_stage_to_regs<W, RS, TR, +1>(sm, stw + tw_offset<P, P::N - 1>(), x, row, t);
    double2 *dst = a.A + m2;
#pragma unroll
    for (int r = 0; r < 16; ++r) dst[(size_t)(t + r * TR) * H] = x[r];
  } else {
    fwd_stages<P, RS, 1, P::N, 16, TR>(sm, stw, row, t, sync);
    for (int k1 = threadIdx.x; k1 < W; k1 += T) a.A[(size_t)k1 * H + m2b] = sm[pad(k1)];
  }
  if (MODE != WIDE_INIT) {
    float em = (float)emax;
#pragma unroll
    for (int o = 16; o; o >>= 1) em = fmaxf(em, __shfl_xor_sync(0xffffffffu, em, o));
    if ((threadIdx.x & 31) == 0) s_err[threadIdx.x >> 5] = em;
    if (out_of_range) atomicOr(&s_fault, 2u);
    sync();
    if (threadIdx.x == 0) {
      float m = 0.f;
      for (int i = 0; i < (T + 31) / 32; ++i) m = fmaxf(m, s_err[i]);
      atomicMax(&a.st->err_bits, __float_as_uint(m));
      if (s_fault) atomicOr(&a.st->fault, s_fault);
    }
  }
}

template <class P, int G, int MODE>
__global__ void __launch_bounds__(wide_threads<P, G>(), min_blocks(wide_threads<P, G>())) wide_static(WideArgs a) {
  wide_body<P, G, MODE, false>(a, 0);
}

// Wide pass for rows of length W = P::L whose radix list starts and ends with
// the same radix R (e.g. 1280 = 8 x 4 x 5 x 8): TR = W/R threads per row, R
// elements each, every stage in shared memory (Stockham, natural order in and
// out, the same list both ways).  The first inverse stage reads straight from
// global memory and the last forward stage writes straight to it; the last
// inverse butterfly of thread t yields elements t + r*TR, which are what it
// rounds and carries and what its first forward butterfly takes, so they stay
// in registers in between.  Fewer elements per thread than wide_body's 16
// keep the registers per thread low and the warps per SM high.  The carry
// arithmetic, the -2 and the warp-by-warp hand-off are those of wide_body
// (colD/colS of the arguments are computed for this TR).
template <class P, int G, int MODE, bool BATCH, class S = CtaSync>
__device__ __forceinline__ void wide_any_body(const WideArgs &a, int blk, S sync = S()) {
  constexpr int W = P::L, R = P::a[0], TR = W / R, T = G * TR;
  static_assert(P::a[P::N - 1] == R, "first and last radix equal: the carried elements stay in registers");
  static_assert(G >= 2, "the rows of an element column in adjacent lanes: whole 32-byte sectors");
  extern __shared__ double2 sm[];
  constexpr int RS = row_slots<W, G>();
  double2 *stw = sm + G * RS;
  __shared__ int s_g;
  __shared__ float s_err[32];
  __shared__ uint32_t s_fault;
  if (threadIdx.x == 0) {
    s_fault = 0;
    s_g = MODE == WIDE_INIT ? (BATCH ? blk : (int)blockIdx.x)
                            : (int)(atomicAdd(&a.st->ticket, 1ull) % (unsigned long long)a.ngroups);
  }
  for (int i = threadIdx.x; i < tw_size<P>(); i += T) cp_async16(&stw[i], &a.stw[i]);
  sync();
  const int g = s_g;
  const int H = a.H;
  const int m2b = g * G;
  const int row = threadIdx.x % G, t = threadIdx.x / G;
  const int m2 = m2b + row;
  const int n = (int)a.n, bb = (int)a.b, qn = (int)a.qn;
  int E0 = __ldg(&a.rowE[2 * m2]) + __ldg(&a.colF[t]);
  int E1 = __ldg(&a.rowE[2 * m2 + 1]) + __ldg(&a.colF[t]);
  const double cwt = __ldg(&a.colW[t]);
  const double W0 = __ldg(&a.rowW[2 * m2]) * cwt * (E0 >= n ? 0.5 : 1.0);
  const double W1 = __ldg(&a.rowW[2 * m2 + 1]) * cwt * (E1 >= n ? 0.5 : 1.0);
  double Wi0 = 0.0, Wi1 = 0.0;
  if (MODE != WIDE_INIT) {
    const double cwit = __ldg(&a.colWi[t]);
    Wi0 = __ldg(&a.rowWi[2 * m2]) * cwit * (E0 >= n ? 2.0 : 1.0);
    Wi1 = __ldg(&a.rowWi[2 * m2 + 1]) * cwit * (E1 >= n ? 2.0 : 1.0);
  }
  if (E0 >= n) E0 -= n;
  if (E1 >= n) E1 -= n;
  const double p2lo = (double)(1 << qn), p2hi = 2.0 * p2lo;
  const double ip2lo = 1.0 / p2lo, ip2hi = 0.5 * ip2lo;
  double2 *rw = sm + row * RS;
  auto ld = [&](int e, int, int) { return rw[pad(e)]; };
  auto st = [&](int e, int, int, double2 v) { rw[pad(e)] = v; };
  double2 x[R];
  double emax = 0.0;
  bool out_of_range = false;
  // everything above reads constant tables only; the state array, the
  // digits and the device state are read after the previous pass completed
  griddep_wait();
  griddep_release();
  if (MODE != WIDE_INIT) {
    // the -2 (bit (offset+1) mod q, CUDALucas.cu:1882-1886) hits at most one
    // word; locate it once: element register r_sub, word w_sub
    const uint32_t off = a.st->offset;
    const uint32_t pos = (off + 1) % a.q;
    const uint32_t dw = (uint32_t)(((unsigned long long)pos * a.n) / a.q);
    const uint32_t sdw = (uint32_t)(((unsigned long long)dw * a.q + a.n - 1) / a.n);
    const double sub = (double)(1u << (pos - sdw));
    int r_sub = -1;
    {
      const uint32_t me = dw >> 1, mm1 = me / (uint32_t)H, mm2 = me - mm1 * (uint32_t)H;
      if ((int)mm2 == m2 && (int)(mm1 % TR) == t) r_sub = (int)(mm1 / TR);
    }
    const bool w_sub = dw & 1;
    // inverse row transform: the first stage straight from global memory,
    // the last into registers (elements t + r*TR)
    const double2 *src = a.A + m2;
    double2 u[R];
    auto ld_first = [&](int e, int, int) { return src[(size_t)e * H]; };
    auto st_reg = [&](int, int, int r, double2 v) { u[r] = v; };
    cp_async_wait_all();  // the stage twiddles, visible after the first stage's barrier
    fall_stages<P, 0, 1, TR, -1, false, false>(stw, t, sync, ld_first, st_reg, ld, st);
    double2 *ks = rw + t;  // ks[r*TR]: element m1 = t + r*TR
    double *gcd = reinterpret_cast<double *>(a.carry);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m1 = t + r * TR;
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const int e0 = E0 - D + (n0 ? n : 0), e1 = E1 - D + (n1 ? n : 0);
      const double t0 = u[r].x * (Wi0 * (n0 ? a.colSi2[r] : a.colSi[r]));
      const double t1 = u[r].y * (Wi1 * (n1 ? a.colSi2[r] : a.colSi[r]));
      double r0 = rint(t0), r1 = rint(t1);
      emax = fmax(emax, fmax(fabs(t0 - r0), fabs(t1 - r1)));
      if (!(fabs(t0) < 0x1p51 && fabs(t1) < 0x1p51)) out_of_range = true;
      if (r == r_sub) {
        if (w_sub) r1 -= sub;
        else r0 -= sub;
      }
      const bool big0 = e0 < bb, big1 = e1 < bb;
      const double P0 = big0 ? p2hi : p2lo, I0 = big0 ? ip2hi : ip2lo;
      const double P1 = big1 ? p2hi : p2lo, I1 = big1 ? ip2hi : ip2lo;
      const double h0 = rnd_int(r0 * I0), l0 = fma(-h0, P0, r0);
      const double h1 = rnd_int(r1 * I1), l1 = fma(-h1, P1, r1);
      const double tt1 = l1 + h0;
      const double k1c = rnd_int(tt1 * I1);
      const double d1p = fma(-k1c, P1, tt1);
      const double co = h1 + k1c;
      ks[r * TR] = make_double2(fma(d1p, 0x1p24, l0), co);
      if (row == G - 1) gcd[(size_t)g * W + m1] = co;
    }
    // hand-off warp by warp, as in wide_body
    const int pred = g == 0 ? a.ngroups - 1 : g - 1;
    constexpr int NW = T / 32;
    static_assert(T % 32 == 0 && NW <= kWarpFlags, "whole warps, one flag each");
    const int warp = threadIdx.x >> 5;
    __syncwarp();
    if ((threadIdx.x & 31) == 0)
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&a.flags[g * kWarpFlags + warp]), "r"(1u) : "memory");
    if (g != 0) {
      if ((threadIdx.x & 31) == 0) {
        uint32_t *f = &a.flags[pred * kWarpFlags + warp];
        if (!wait_flag(f)) atomicOr(&s_fault, 1u);
        *f = 0;
      }
      __syncwarp();
    } else {
      sync();
      if (threadIdx.x == 0) {
        for (int w = 0; w < NW; ++w) {
          uint32_t *f = &a.flags[pred * kWarpFlags + w];
          if (!wait_flag(f)) s_fault |= 1u;
          *f = 0;
        }
      }
      sync();
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m1 = t + r * TR;
      const double cin = row > 0 ? sm[(row - 1) * RS + m1].y
                                 : __ldcg(&gcd[(size_t)pred * W + (g == 0 ? (m1 == 0 ? W - 1 : m1 - 1) : m1)]);
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const int e0 = E0 - D + (n0 ? n : 0);
      const bool big0 = e0 < bb;
      const double P0 = big0 ? p2hi : p2lo, I0 = big0 ? ip2hi : ip2lo;
      const double pk = ks[r * TR].x;
      const double d1p = rnd_int(pk * 0x1p-24), l0 = fma(-d1p, 0x1p24, pk);
      const double tt0 = l0 + cin;
      const double k0 = rnd_int(tt0 * I0);
      const double d0 = fma(-k0, P0, tt0);
      const double d1 = d1p + k0;
      if (MODE == WIDE_REPORT) {
        const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
        a.xint[j0] = (int32_t)d0;
        a.xint[j0 + 1] = (int32_t)d1;
      }
      x[r] = make_double2(d0 * (W0 * (n0 ? a.colS2[r] : a.colS[r])), d1 * (W1 * (n1 ? a.colS2[r] : a.colS[r])));
    }
  } else {
    cp_async_wait_all();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int m1 = t + r * TR;
      const int D = a.colD[r];
      const bool n0 = E0 < D, n1 = E1 < D;
      const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
      x[r] = make_double2((double)a.xint[j0] * (W0 * (n0 ? a.colS2[r] : a.colS[r])),
                          (double)a.xint[j0 + 1] * (W1 * (n1 ? a.colS2[r] : a.colS[r])));
    }
  }
  // forward row transform: the first stage from registers (its barrier
  // orders the carry reads above before the row is rewritten), the last
  // straight to global memory
  double2 *dst = a.A + m2;
  auto ld_reg = [&](int, int, int r) { return x[r]; };
  auto st_last = [&](int e, int, int, double2 v) { dst[(size_t)e * H] = v; };
  fall_stages<P, 0, 1, TR, +1, true, false>(stw, t, sync, ld_reg, st_last, ld, st);
  if (MODE != WIDE_INIT) {
    float em = (float)emax;
#pragma unroll
    for (int o = 16; o; o >>= 1) em = fmaxf(em, __shfl_xor_sync(0xffffffffu, em, o));
    if ((threadIdx.x & 31) == 0) s_err[threadIdx.x >> 5] = em;
    if (out_of_range) atomicOr(&s_fault, 2u);
    sync();
    if (threadIdx.x == 0) {
      float m = 0.f;
      for (int i = 0; i < (T + 31) / 32; ++i) m = fmaxf(m, s_err[i]);
      atomicMax(&a.st->err_bits, __float_as_uint(m));
      if (s_fault) atomicOr(&a.st->fault, s_fault);
    }
  }
}

template <class P, int G>
__host__ __device__ constexpr int wide_any_threads() { return G * (P::L / P::a[0]); }

template <class P, int G, int MINB, int MODE>
__global__ void __launch_bounds__(wide_any_threads<P, G>(), MINB) wide_any(WideArgs a) {
  wide_any_body<P, G, MODE, false>(a, 0);
}

// ---- batched launches: one launch runs a pass for every member of a length
// class (members of one FFT length share the kernel); blockIdx.x = member *
// units + unit.  A member's arguments are copied from the class's device
// array into shared memory before anything else; they are constant for the
// life of the batch, so this may overlap the previous pass (PDL).
template <class Args>
__device__ __forceinline__ const Args &member_args(const Args *arr, int m, Args *sa) {
  static_assert(sizeof(Args) % 8 == 0, "copied as 64-bit words");
  const uint64_t *src = reinterpret_cast<const uint64_t *>(&arr[m]);
  uint64_t *dst = reinterpret_cast<uint64_t *>(sa);
  for (int i = threadIdx.x; i < (int)(sizeof(Args) / 8); i += blockDim.x) dst[i] = __ldg(&src[i]);
  __syncthreads();
  return *sa;
}

template <class P>
__global__ void __launch_bounds__(tall_threads<P>(), min_blocks(tall_threads<P>()))
    tall_static_batch(const TallArgs *arr, int units) {
  __shared__ __align__(16) TallArgs sa;
  const int m = blockIdx.x / units;
  const TallArgs &a = member_args(arr, m, &sa);
  tall_body<P>(a, blockIdx.x - m * units);
}

template <class P, int TC, int PP>
__global__ void __launch_bounds__(2 * PP * TC, min_blocks(2 * PP * TC)) tall_any_batch(const TallArgs *arr, int units) {
  __shared__ __align__(16) TallArgs sa;
  const int m = blockIdx.x / units;
  const TallArgs &a = member_args(arr, m, &sa);
  tall_any_body<P, TC, PP>(a, blockIdx.x - m * units);
}

template <class P, int G>
__global__ void __launch_bounds__(wide_threads<P, G>(), min_blocks(wide_threads<P, G>()))
    wide_static_batch(const WideArgs *arr, int units) {
  __shared__ __align__(16) WideArgs sa;
  const int m = blockIdx.x / units;
  const WideArgs &a = member_args(arr, m, &sa);
  wide_body<P, G, WIDE_ITER, true>(a, blockIdx.x - m * units);
}

template <class P, int G, int MINB>
__global__ void __launch_bounds__(wide_any_threads<P, G>(), MINB) wide_any_batch(const WideArgs *arr, int units) {
  __shared__ __align__(16) WideArgs sa;
  const int m = blockIdx.x / units;
  const WideArgs &a = member_args(arr, m, &sa);
  wide_any_body<P, G, WIDE_ITER, true>(a, blockIdx.x - m * units);
}

// ---- fused iterations for short lengths ---------------------------------
// One cooperative launch runs `iters` iterations: every CTA takes part in
// both passes, looping over their units, and the passes are separated by
// grid-wide barriers instead of kernel boundaries, so a length whose passes
// are a few microseconds of work each no longer pays two launches per
// iteration.  The block has max(T1, T2) threads; a pass whose CTA shape is
// smaller runs on the first threads with a named barrier.

// Grid-wide barrier (all CTAs are co-resident: cooperative launch).  The
// fences around the arrival make every CTA's writes before the barrier
// visible to every CTA's reads after it.  The wait is bounded: on expiry it
// sets fault bit 0 and returns false.
__device__ __forceinline__ bool grid_sync(DevState *st, unsigned nblocks) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned g;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(&st->bar_gen) : "memory");
    __threadfence();
    int ok = 1;
    if (atomicAdd(&st->bar_count, 1u) == nblocks - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&st->bar_gen), "r"(g + 1u) : "memory");
    } else {
      ok = 0;
      for (int it = 0; it < (1 << 24); ++it) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&st->bar_gen) : "memory");
        if (v != g) {
          ok = 1;
          break;
        }
        __nanosleep(it < 64 ? 32 : 256);
      }
      if (!ok) atomicOr(&st->fault, 1u);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Tall pass of the fused kernel: tall_body (TC == 0) or tall_any_body.
template <class PT, int TC, int PP>
struct FusedTall {
  static constexpr int threads = TC ? 2 * PP * TC : tall_threads<PT>();
  template <class S>
  __device__ __forceinline__ static void run(const TallArgs &a, int u, S sync) {
    if constexpr (TC) tall_any_body<PT, TC, PP, S>(a, u, sync);
    else tall_body<PT, S>(a, u, sync);
  }
};

template <class PW, int G, class TP>
__host__ __device__ constexpr int fused_threads() {
  return wide_threads<PW, G>() > TP::threads ? wide_threads<PW, G>() : TP::threads;
}

template <class PW, int G, class TP>
__global__ void __launch_bounds__(fused_threads<PW, G, TP>(), 1)
    fused_iters(TallArgs ta, WideArgs wa, uint32_t iters, int tall_units) {
  constexpr int TPB = fused_threads<PW, G, TP>(), T1 = wide_threads<PW, G>(), T2 = TP::threads;
  static_assert((T1 == TPB || T1 % 32 == 0) && (T2 == TPB || T2 % 32 == 0),
                "a pass on part of the CTA needs whole warps (named barrier)");
  const int wide_units = wa.ngroups;
  for (uint32_t it = 0; it < iters; ++it) {
    for (int u = blockIdx.x; u < tall_units; u += gridDim.x) {
      if constexpr (T2 == TPB) TP::run(ta, u, CtaSync());
      else if (threadIdx.x < T2) TP::run(ta, u, PartSync{1, T2});
      __syncthreads();  // the next unit reuses the shared memory
    }
    if (!grid_sync(ta.st, gridDim.x)) return;
    for (int u = blockIdx.x; u < wide_units; u += gridDim.x) {
      if constexpr (T1 == TPB) wide_body<PW, G, WIDE_ITER, false>(wa, u, CtaSync());
      else if (threadIdx.x < T1) wide_body<PW, G, WIDE_ITER, false>(wa, u, PartSync{1, T1});
      __syncthreads();
    }
    if (!grid_sync(ta.st, gridDim.x)) return;
  }
}

