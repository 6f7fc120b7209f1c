// Cluster-resident iterations for short lengths (N = W * H complex elements
// small enough to live in the shared memory of one thread-block cluster).
//
// Short lengths are latency bound: at 12K two launches per iteration, the
// loads of the state from L2 and the carry flags through L2 cost far more
// than the arithmetic.  Here one launch runs any number of iterations; the
// state stays in the distributed shared memory of the cluster's C CTAs, and
// the passes are separated by hardware cluster barriers:
//
//   * CTA `rank` owns the column pairs p = rank*PPC .. rank*PPC+PPC-1 (columns
//     kA = p, kB = W-p; pair 0 holds the self-paired columns 0 and W/2), each
//     column H elements in its own shared memory (padded slots), and runs
//     their tall pass: twiddle w_N^(k1*m2) (folded into the first stage's
//     loads), H-point FFT, pairing and squaring, inverse FFT whose last stage
//     applies the conjugate twiddle and stores every element straight into
//     the row buffer of the CTA that owns its row (the tall_any arithmetic);
//   * cluster barrier;
//   * CTA `rank` also owns the rows m2 = rank*RPC .. rank*RPC+RPC-1 (ranks
//     past H/RPC own none).  Its wide pass runs the inverse row FFT on its
//     row buffers, unweights, rounds, subtracts 2 and splits the carries
//     (the wide_static arithmetic); the carries of its last row are stored
//     into the carry row of the next CTA;
//   * the first row of each CTA waits for those carries (rank 0 the carries
//     of row H-1, shifted by one element: the 2^q == 1 wrap) on an mbarrier
//     that the previous CTA arrives on once it has stored them (a pairwise
//     hand-off, not a cluster barrier); the digits are reweighted and
//     transformed forward, and the last stage stores every element straight
//     into the column buffer of its column owner;
//   * cluster barrier.
//
// Every transfer between CTAs is a store into the other CTA's shared memory
// (no remote loads, whose latency would sit on the critical path); the
// cluster barrier that follows, or for the carries the mbarrier arrive with
// release semantics, makes it visible.  A row is short and its pass
// latency bound, so it is spread over TWR threads (a few elements each) and
// transformed in shared memory with a radix list of small radices (Stockham
// stages, natural order in and out); the elements a thread rounds and
// carries are exactly the outputs of its last inverse butterfly and the
// inputs of its first forward one, so they stay in registers in between.
// The weights are formed per element from the row and column tables.
//
// An element is touched by its column owner in the tall pass and by its row
// owner in the wide pass only, so the three barriers order every access.
// The state is loaded from HBM at the start of the launch and stored back at
// the end, in the layout of the two-launch path (A[k1][m2]); the shift
// doubles every iteration in a register of every thread.  The barriers are
// taken by every thread of every CTA the same number of times, and no CTA
// touches another's shared memory after the last one.
//
// The digits equal those of the two-launch path (the rounded values agree
// while the roundoff error stays below 0.5); the roundoff maximum differs in
// its last bits, the row transforms being factored differently.

template <class PR, int TWR, class PT, int TC, int C, int RPC>
struct ClusterCfg {
  static constexpr int W = PR::L, H = PT::L;
  static constexpr int EPR = W / TWR;                    // elements of a row per thread
  static constexpr int PPC = W / 2 / C;                  // column pairs per CTA
  static constexpr int CS = col_slots<H>();              // padded column
  static constexpr int RS = col_slots<W>() + 1;          // padded row (odd stride of pairs of banks)
  static constexpr int PS = H + 1;                       // pairing twiddles per pair
  static constexpr int TT = 2 * PPC * TC;                // tall-pass threads
  static constexpr int TW = RPC * TWR;                   // wide-pass threads
  static constexpr int T = TT > TW ? TT : TW;
  static constexpr int ROWCTAS = H / RPC;                // CTAs that own rows
  // dynamic shared memory (double2 entries)
  static constexpr int o_stw = RPC * RS;                 // row stage twiddles
  static constexpr int o_stt = o_stw + tw_size<PR>();    // column stage twiddles
  static constexpr int o_col = o_stt + tw_size<PT>();    // the owned columns (state)
  static constexpr int o_ctw = o_col + 2 * PPC * CS;     // w_N^(k1*m2) of the owned columns
  static constexpr int o_ptw = o_ctw + 2 * PPC * H;      // pairing twiddles
  static constexpr int o_cwt = o_ptw + PPC * PS;         // column weights (2^(colF/n), 2^(-colF/n))
  static constexpr int o_cf = o_cwt + W;                 // column exponents colF (W int32)
  static constexpr int o_cin = o_cf + W / 4;             // carries into the first row (W doubles)
  static constexpr int total = o_cin + W / 2;
  static_assert(W % 4 == 0 && (W / 2) % C == 0 && PPC >= 1, "whole column pairs per CTA");
  static_assert(W % TWR == 0 && TWR % 32 == 0, "whole warps per row");
  static_assert(H % RPC == 0 && ROWCTAS <= C, "whole row groups, at most one per CTA");
  static_assert(TT == T || TT % 32 == 0, "a tall pass on part of the CTA needs whole warps");
  static_assert(PR::N <= 4, "the host keeps four radices of the row list");
  static_assert(W / PR::a[0] == TWR && W / PR::a[PR::N - 1] == TWR,
                "first and last row stages: one butterfly per thread, elements t + j*TWR");
};

// floor(x / d) for x < 2^58 and d < 2^31: an FP64 estimate (off by at most
// one, its relative error is a few 2^-53 and the quotient is below 2^31),
// then one exact correction step in integers.
__device__ __forceinline__ uint32_t udiv_est(unsigned long long x, uint32_t d, double inv_d) {
  unsigned long long e = (unsigned long long)((double)x * inv_d);
  if (e * d > x) --e;
  else if ((e + 1) * d <= x) ++e;
  return (uint32_t)e;
}

// Point-to-point hand-off between two CTAs of the cluster through an
// mbarrier in the receiver's shared memory: the sender's stores into the
// receiver, a CTA barrier, then one release arrive on the receiver's
// barrier; the receiver waits with acquire at cluster scope.  The wait is
// bounded: on expiry it returns false (the caller sets the timeout fault bit
// and goes on, so every later barrier is still taken).
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ uint32_t mbar_remote(uint64_t *bar, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_addr(bar)), "r"(rank));
  return a;
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t remote) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (int k = 0; k < (1 << 22); ++k) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Column k1 held in local column slot lc of CTA `rank`.
template <class CF>
__device__ __forceinline__ int cluster_col_k1(int rank, int lc) {
  const int p = rank * CF::PPC + (lc >> 1);
  return (lc & 1) ? (p == 0 ? CF::W / 2 : CF::W - p) : p;
}

// Element (k1, m2) in the shared memory of its column owner.
template <class CF>
__device__ __forceinline__ double2 *cluster_slot(cooperative_groups::cluster_group &cl, double2 *cols, int k1, int m2) {
  const int side = k1 >= CF::W / 2;
  const int p = side ? (k1 == CF::W / 2 ? 0 : CF::W - k1) : k1;
  const int lc = 2 * (p % CF::PPC) + side;
  return cl.map_shared_rank(cols + lc * CF::CS + pad(m2), (unsigned)(p / CF::PPC));
}

template <class PR, int TWR, class PT, int TC, int C, int RPC>
__global__ void __launch_bounds__(ClusterCfg<PR, TWR, PT, TC, C, RPC>::T, 1)
    cluster_iters(TallArgs ta, WideArgs wa, const double2 *stwr, uint32_t iters, int report) {
  // stwr: stage twiddles of the row list PR, then of the column list PT
  using CF = ClusterCfg<PR, TWR, PT, TC, C, RPC>;
  constexpr int W = CF::W, H = CF::H, EPR = CF::EPR, PPC = CF::PPC, CS = CF::CS, RS = CF::RS, PS = CF::PS;
  constexpr int T = CF::T, TT = CF::TT, TW = CF::TW;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ double2 sm[];
  __shared__ float s_err[32];
  __shared__ uint32_t s_fault;
  __shared__ __align__(8) uint64_t s_cbar;  // the previous CTA's carries have arrived
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x;
  double2 *rows = sm;
  double2 *stw = sm + CF::o_stw, *stt = sm + CF::o_stt;
  double2 *cols = sm + CF::o_col, *ctw = sm + CF::o_ctw, *ptw = sm + CF::o_ptw;
  double2 *cwt = sm + CF::o_cwt;
  int *cf = reinterpret_cast<int *>(sm + CF::o_cf);
  double *cin = reinterpret_cast<double *>(sm + CF::o_cin);

  // ---- set-up: tables, twiddles of the owned columns, the owned state
  if (tid == 0) {
    s_fault = 0;
    mbar_init(&s_cbar, 1);  // one arrive per iteration: the previous CTA's
  }
  for (int i = tid; i < tw_size<PR>(); i += T) stw[i] = stwr[i];
  for (int i = tid; i < tw_size<PT>(); i += T) stt[i] = stwr[tw_size<PR>() + i];
  for (int i = tid; i < W; i += T) {
    cwt[i] = make_double2(wa.colW[i], wa.colWi[i]);
    cf[i] = wa.colF[i];
  }
  for (int i = tid; i < 2 * PPC * H; i += T) {
    const int lc = i / H, m2 = i - lc * H;
    const int k1 = cluster_col_k1<CF>(rank, lc);
    ctw[i] = omegaN(ta.thi, ta.tlo, ta.ts, ta.tmask, k1 * m2);
    cols[lc * CS + pad(m2)] = ta.A[(size_t)k1 * H + m2];
  }
  for (int i = tid; i < PPC * PS; i += T) {
    const int pl = i / PS, j = i - pl * PS;
    const int p = rank * PPC + pl;
    int e;
    if (p != 0) e = j < H ? p + W * j : 0;
    else e = j <= H / 2 ? W * j : W / 2 + W * (j - H / 2 - 1);
    ptw[i] = omegaN(ta.thi, ta.tlo, ta.ts, ta.tmask, e);
  }

  // ---- wide-pass constants of this thread: row m2, elements t + j*TWR
  const bool wide = rank < CF::ROWCTAS && tid < TW;
  const int row = tid / TWR, t = tid - (tid / TWR) * TWR;
  const int m2 = rank * RPC + row;
  const int n = (int)wa.n, bb = (int)wa.b, qn = (int)wa.qn;
  const uint32_t q = wa.q, un = wa.n;
  const double inv_q = 1.0 / (double)q, inv_n = 1.0 / (double)un;
  int rE0 = 0, rE1 = 0;
  double rW0 = 0.0, rW1 = 0.0, rWi0 = 0.0, rWi1 = 0.0;
  if (wide) {
    rE0 = wa.rowE[2 * m2];
    rE1 = wa.rowE[2 * m2 + 1];
    rW0 = wa.rowW[2 * m2];
    rW1 = wa.rowW[2 * m2 + 1];
    rWi0 = wa.rowWi[2 * m2];
    rWi1 = wa.rowWi[2 * m2 + 1];
  }
  const double p2lo = (double)(1 << qn), p2hi = 2.0 * p2lo;
  const double ip2lo = 1.0 / p2lo, ip2hi = 0.5 * ip2lo;
  // the carries of the last row go to the next CTA's carry row (into rank 0
  // shifted by one element)
  const bool wrap = rank == CF::ROWCTAS - 1;
  double *next_cin = cl.map_shared_rank(cin, (unsigned)(wrap ? 0 : rank + 1));
  const uint32_t next_cbar = mbar_remote(&s_cbar, (unsigned)(wrap ? 0 : rank + 1));
  uint32_t off = ta.st->offset;
  double emax = 0.0;
  bool out_of_range = false;
  double2 *rw = rows + row * RS;

  // tall-pass thread: column `col` (local slot) of pair pl, thread tc of TC
  const int col = tid / TC, tc = tid - (tid / TC) * TC;
  const int pl = col >> 1;
  const bool special = rank == 0 && pl == 0;
  const int my_k1 = cluster_col_k1<CF>(rank, col < 2 * PPC ? col : 0);
  using SyncT = typename std::conditional<TT == T, CtaSync, PartSync>::type;
  using SyncW = typename std::conditional<TW == T, CtaSync, PartSync>::type;
  SyncT syncT;
  SyncW syncW;
  if constexpr (TT != T) syncT = SyncT{1, TT};
  if constexpr (TW != T) syncW = SyncW{2, TW};

  cl.sync();  // every CTA of the cluster is running and has its state

  for (uint32_t it = 0; it < iters; ++it) {
    // CUDALucas.cu:1882: offset <- 2*offset mod q, once per iteration
    off = 2u * off >= q ? 2u * off - q : 2u * off;
    // ---------------------------------------------------------- tall pass
    if (tid < TT) {
      double2 *cc = cols + col * CS;
      const double2 *cw = ctw + col * H;
      auto ld = [&](int e, int, int) { return cc[pad(e)]; };
      auto st = [&](int e, int, int, double2 v) { cc[pad(e)] = v; };
      auto ld_tw = [&](int e, int, int) { return cmul(cc[pad(e)], cw[e]); };
      fall_stages<PT, 0, 1, TC, +1, true, true>(stt, tc, syncT, ld_tw, st, ld, st);
      const int ti = tid - 2 * pl * TC;
      double2 *ra = cols + 2 * pl * CS, *rb = ra + CS;
      const double2 *pw = ptw + pl * PS;
      if (!special) {
        for (int k2 = ti; k2 < H; k2 += 2 * TC) {
          double2 za = ra[pad(k2)], zb = rb[pad(H - 1 - k2)];
          pair_square(za, zb, pw[k2]);
          ra[pad(k2)] = za;
          rb[pad(H - 1 - k2)] = zb;
        }
      } else {
        for (int i = ti; i <= H / 2; i += 2 * TC) {
          const int p2 = (H - i) % H;
          double2 za = ra[pad(i)], zb = ra[pad(p2)];
          pair_square(za, zb, pw[i]);
          ra[pad(i)] = za;
          if (p2 != i) ra[pad(p2)] = zb;
        }
        for (int i = ti; i < H / 2; i += 2 * TC) {
          double2 za = rb[pad(i)], zb = rb[pad(H - 1 - i)];
          pair_square(za, zb, pw[H / 2 + 1 + i]);
          rb[pad(i)] = za;
          rb[pad(H - 1 - i)] = zb;
        }
      }
      syncT();
      // the last inverse stage: conjugate twiddle, then element (my_k1, e)
      // into the row buffer of the CTA that owns row e
      auto st_push = [&](int e, int, int, double2 v) {
        *cl.map_shared_rank(rows + (e % RPC) * RS + pad(my_k1), (unsigned)(e / RPC)) = cmulc(v, cw[e]);
      };
      fall_stages<PT, 0, 1, TC, -1, true, false>(stt, tc, syncT, ld, st_push, ld, st);
    }
    cl.sync();  // every row buffer holds its row
    // ---------------------------------------------------------- wide pass
    if (wide) {
      // the -2 (bit (offset+1) mod q, CUDALucas.cu:1882-1886): element
      // j_sub, word w_sub of the thread that holds it
      const uint32_t pos = off + 1 == q ? 0u : off + 1;
      const uint32_t dw = udiv_est((unsigned long long)pos * un, q, inv_q);
      const uint32_t sdw = udiv_est((unsigned long long)dw * q + un - 1, un, inv_n);
      const double sub = (double)(1u << (pos - sdw));
      int j_sub = -1;
      {
        const uint32_t me = dw >> 1, mm1 = me / (uint32_t)H, mm2 = me - mm1 * (uint32_t)H;
        if ((int)mm2 == m2 && (int)(mm1 % TWR) == t) j_sub = (int)(mm1 / TWR);
      }
      const bool w_sub = dw & 1;
      // inverse row transform; its last stage leaves elements t + j*TWR in u[j]
      double2 u[EPR];
      auto ld = [&](int e, int, int) { return rw[pad(e)]; };
      auto st = [&](int e, int, int, double2 v) { rw[pad(e)] = v; };
      auto st_reg = [&](int, int, int r, double2 v) { u[r] = v; };
      fall_stages<PR, 0, 1, TWR, -1, true, false>(stw, t, syncW, ld, st_reg, ld, st);
#pragma unroll
      for (int j = 0; j < EPR; ++j) {
        const int m1 = t + j * TWR;
        const int cfm = cf[m1];
        const double cwi = cwt[m1].y;
        int e0 = rE0 + cfm, e1 = rE1 + cfm;
        const bool f0 = e0 >= n, f1 = e1 >= n;
        if (f0) e0 -= n;
        if (f1) e1 -= n;
        const double t0 = u[j].x * (rWi0 * cwi * (f0 ? 2.0 : 1.0));
        const double t1 = u[j].y * (rWi1 * cwi * (f1 ? 2.0 : 1.0));
        double r0 = rint(t0), r1 = rint(t1);
        emax = fmax(emax, fmax(fabs(t0 - r0), fabs(t1 - r1)));
        // at 2^51 and above (or NaN) a double has no fraction bits left for
        // the roundoff reading, and the exact carry split no longer holds
        if (!(fabs(t0) < 0x1p51 && fabs(t1) < 0x1p51)) out_of_range = true;
        if (j == j_sub) {
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
        rw[m1] = make_double2(fma(d1p, 0x1p24, l0), co);
        if (row == RPC - 1) next_cin[wrap ? (m1 + 1 == W ? 0 : m1 + 1) : m1] = co;
      }
      // the carries of this CTA's rows are in place (the next row reads them
      // below); those of the last row go to the next CTA with one release
      syncW();
      if (tid == 0) mbar_arrive_remote(next_cbar);
    }
    if (wide) {
      // the first row waits for the previous CTA's carries (the only
      // dependence between CTAs inside the wide pass)
      if (row == 0 && !mbar_wait(&s_cbar, it & 1u)) atomicOr(&s_fault, 1u);
      const bool last_it = report && it + 1 == iters;
      double2 x[EPR];
#pragma unroll
      for (int j = 0; j < EPR; ++j) {
        const int m1 = t + j * TWR;
        const double c_in = row > 0 ? rows[(row - 1) * RS + m1].y : cin[m1];
        const int cfm = cf[m1];
        const double cw = cwt[m1].x;
        int e0 = rE0 + cfm;
        const bool f0 = e0 >= n, f1 = rE1 + cfm >= n;
        if (f0) e0 -= n;
        const bool big0 = e0 < bb;
        const double P0 = big0 ? p2hi : p2lo, I0 = big0 ? ip2hi : ip2lo;
        const double pk = rw[m1].x;
        const double d1p = rnd_int(pk * 0x1p-24), l0 = fma(-d1p, 0x1p24, pk);
        const double tt0 = l0 + c_in;
        const double k0 = rnd_int(tt0 * I0);
        const double d0 = fma(-k0, P0, tt0);
        const double d1 = d1p + k0;
        if (last_it) {
          const uint32_t j0 = 2u * ((uint32_t)m1 * (uint32_t)H + (uint32_t)m2);
          wa.xint[j0] = (int32_t)d0;
          wa.xint[j0 + 1] = (int32_t)d1;
        }
        x[j] = make_double2(d0 * (rW0 * cw * (f0 ? 0.5 : 1.0)), d1 * (rW1 * cw * (f1 ? 0.5 : 1.0)));
      }
      // forward row transform: the first stage takes x[j] from registers
      // (its barrier orders the carry reads above before the row is
      // rewritten); the last stores element (k1, m2) into its column owner
      auto ld = [&](int e, int, int) { return rw[pad(e)]; };
      auto st = [&](int e, int, int, double2 v) { rw[pad(e)] = v; };
      auto ld_reg = [&](int, int, int r) { return x[r]; };
      auto st_push = [&](int e, int, int, double2 v) { *cluster_slot<CF>(cl, cols, e, m2) = v; };
      fall_stages<PR, 0, 1, TWR, +1, true, false>(stw, t, syncW, ld_reg, st_push, ld, st);
    }
    cl.sync();  // the state is whole again
  }

  // ---- store the owned columns, the shift, the roundoff maximum
  for (int i = tid; i < 2 * PPC * H; i += T) {
    const int lc = i / H, m = i - lc * H;
    ta.A[(size_t)cluster_col_k1<CF>(rank, lc) * H + m] = cols[lc * CS + pad(m)];
  }
  if (rank == 0 && tid == 0) ta.st->offset = off;
  if (tid < TW) {
    float em = (float)emax;
#pragma unroll
    for (int o = 16; o; o >>= 1) em = fmaxf(em, __shfl_xor_sync(0xffffffffu, em, o));
    if ((tid & 31) == 0) s_err[tid >> 5] = em;
  }
  if (out_of_range) atomicOr(&s_fault, 2u);
  __syncthreads();
  if (tid == 0 && rank < CF::ROWCTAS) {
    float m = 0.f;
    for (int i = 0; i < TW / 32; ++i) m = fmaxf(m, s_err[i]);
    atomicMax(&wa.st->err_bits, __float_as_uint(m));
    if (s_fault) atomicOr(&wa.st->fault, s_fault);
  }
}
