/*
 * llb200.h -- C ABI of the B200 Lucas-Lehmer engine (libllb200.so).
 *
 * The engine replaces the per-iteration squaring of CUDALucas v2.06:
 *   float lucas_square(int q, int n, int iter, int last, int *offset,
 *                      float *maxerr, int error_flag)      CUDALucas.cu:1869
 * which works on module-global device buffers set up by init_lucas
 * (CUDALucas.cu:1344) and torn down by close_lucas (CUDALucas.cu:1415).
 * Here every exponent under test is an opaque context that owns its device
 * buffers and its CUDA stream, so several contexts can live in one process.
 * No function calls exit(); every failure is a status code.
 *
 * Plain C types only: pointers are host pointers unless stated otherwise.
 */
#ifndef LLB200_H
#define LLB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LL_OK = 0,
  LL_ERR_ARG = 1,       /* bad argument (exponent, length, pointer, size)   */
  LL_ERR_SHAPE = 2,     /* no supported FFT decomposition for this length   */
  LL_ERR_CUDA = 3,      /* CUDA runtime error (see ll_last_error)           */
  LL_ERR_NOMEM = 4,     /* device or host allocation failed                 */
  LL_ERR_STATE = 5,     /* call out of order (e.g. digits not current)      */
  LL_ERR_TIMEOUT = 6,   /* a bounded device-side wait gave up               */
  LL_ERR_INJECTED = 7   /* failure injected through ll_debug_inject_failure */
} ll_status;

/* Flags of ll_step.  LL_REPORT mirrors bit 0 of lucas_square's error_flag
 * (digits written on the last iteration, CUDALucas.cu:1929); LL_ERRCHK
 * mirrors bit 1 (max roundoff error read back, CUDALucas.cu:1973-1978). */
#define LL_REPORT 1u
#define LL_ERRCHK 2u
/* LL_ASYNC: only enqueue, even with LL_REPORT or LL_ERRCHK.  With LL_REPORT
 * the digits become readable once the stream has finished (ll_read_digits
 * waits for it); the roundoff maximum keeps accumulating on the device until
 * the next call that reads it back. */
#define LL_ASYNC 4u

typedef struct ll_ctx ll_ctx;

/* Optional launch shape.  Zero fields are chosen by the engine. */
typedef struct {
  int32_t width;        /* W: row-transform length (complex elements)       */
  int32_t rows_per_cta; /* G: rows handled by one CTA of the wide pass      */
  int32_t threads_wide; /* threads per CTA of the wide pass                 */
  int32_t threads_tall; /* threads per CTA of the tall pass                 */
  int32_t graph_iters;  /* iterations captured per CUDA graph (0 = auto)    */
  int32_t kernels;      /* LL_KERNELS_* flags (0 = the engine's choice)     */
  int32_t cluster_variant; /* among the cluster-resident kernels of the
                              length: 0 = the first that fits the device,
                              v > 0 = the v-th entry (0-based)               */
  int32_t reserved;
} ll_tuning;

/* ll_tuning.kernels: LL_KERNELS_GENERIC forces the generic (runtime-plan)
 * kernels; LL_KERNELS_FUSED runs the plain iterations of the short lengths
 * that have a fused cooperative kernel (12K, 14K, 56K) as one launch with
 * grid barriers between the passes, instead of two launches per iteration
 * (measured slower at 12K and 14K, equal at 56K, so not the default);
 * LL_KERNELS_NO_PREFETCH turns off the L2 prefetch that lengths larger than
 * L2 use.  Short lengths with a cluster-resident kernel (8K, 10K, 12K, 14K,
 * 16K, 18K, 20K, 32K, 36K, 42K, 48K, 56K) run each ll_step as one launch of
 * one thread-block cluster whose shared memory holds the whole state;
 * LL_KERNELS_NO_CLUSTER turns that off (two launches per iteration),
 * LL_KERNELS_CLUSTER8 keeps to the portable cluster size of 8 CTAs. */
#define LL_KERNELS_GENERIC 1
#define LL_KERNELS_FUSED 2
#define LL_KERNELS_NO_PREFETCH 4  /* no L2 prefetch of the next wave's data */
#define LL_KERNELS_NO_CLUSTER 8   /* no cluster-resident iterations */
#define LL_KERNELS_CLUSTER8 16    /* clusters of at most 8 CTAs */
#define LL_KERNELS_ALT_WIDE 32    /* the alternative row kernel where a length has one
                                     (rows in shared memory, 8 elements per thread) */

/* Creates a context for exponent q at FFT length n (FP64 words) on `device`.
 * With tuning NULL (or all zero) the engine chooses the launch: for some
 * lengths from a built-in table of shapes measured fastest on the B200.
 * Replaces alloc_gpu_mem + write_gpu_data (CUDALucas.cu:1096, :1125).
 * n must be even, n/2 must factor into a supported W x H split, q > n. */
ll_status ll_create(int device, uint32_t q, uint32_t n, const ll_tuning *tuning,
                    ll_ctx **out);

/* Releases the context (CUDALucas.cu:1415 close_lucas). NULL is a no-op. */
void ll_destroy(ll_ctx *ctx);

/* Starts a fresh test: s0 = 4 stored as 4*2^offset (CUDALucas.cu:1254-1262
 * init_x with the offset given instead of rand() % q). */
ll_status ll_start(ll_ctx *ctx, uint32_t offset);

/* Loads n balanced digits (word j holds floor(q/n) or floor(q/n)+1 bits) of
 * x = s * 2^offset mod 2^q-1 (CUDALucas.cu:1254-1278 init_x/apply_weights
 * on a resumed test). */
ll_status ll_load_digits(ll_ctx *ctx, const int32_t *digits, uint32_t offset);

/* Runs `iters` LL iterations (iters x lucas_square, CUDALucas.cu:1869).
 * LL_REPORT: digits of the final state become readable by ll_read_digits.
 * LL_REPORT or LL_ERRCHK (without LL_ASYNC): waits for the GPU and stores
 * the max roundoff error seen since the last read in *max_err (may be NULL).
 * Without either flag, or with LL_ASYNC, the call only enqueues work. */
ll_status ll_step(ll_ctx *ctx, uint32_t iters, uint32_t flags, float *max_err);

/* Copies the n digits written by the last LL_REPORT step (or the last
 * load/start) and the matching offset (CUDALucas.cu:2963 g_xint D2H). */
ll_status ll_read_digits(ll_ctx *ctx, int32_t *digits, uint32_t *offset);

/* Res64 of the current state (find_residue, CUDALucas.cu:1491); requires
 * current digits like ll_read_digits. */
ll_status ll_res64(ll_ctx *ctx, uint64_t *res64);

/* Device-resident checkpoint (no counterpart in the reference, which keeps
 * its restart point packed on the host, CUDALucas.cu:2963-2980).
 * ll_device_checkpoint enqueues a device-to-device copy of the digits the
 * last LL_REPORT step wrote (LL_ASYNC included) into a buffer the context
 * owns (4n bytes, allocated by the first call) and remembers their offset.
 * ll_device_restore enqueues the reload of the state from that copy (as
 * ll_load_digits does from the host) and returns the restored offset;
 * neither call waits for the GPU. */
ll_status ll_device_checkpoint(ll_ctx *ctx);
ll_status ll_device_restore(ll_ctx *ctx, uint32_t *offset);

/* Device memory a context for (q, n) allocates, in bytes (its state array,
 * digits, carry rows, flags and tables; the device checkpoint adds 4n), or
 * 0 if the length is not supported.  Host-only. */
uint64_t ll_context_bytes(uint32_t q, uint32_t n, const ll_tuning *tuning);

/* Waits for all queued work of the context. */
ll_status ll_sync(ll_ctx *ctx);

/* Non-blocking: 1 while queued work of the context is still running, 0 when
 * it is idle, -1 on a CUDA error (the serving loop polls with this). */
int32_t ll_busy(ll_ctx *ctx);

/* Properties of a context. */
uint32_t ll_exponent(const ll_ctx *ctx);
uint32_t ll_fft_length(const ll_ctx *ctx);
uint32_t ll_offset(const ll_ctx *ctx);
void *ll_stream(const ll_ctx *ctx);           /* the context's cudaStream_t */
void ll_shape(const ll_ctx *ctx, int32_t *width, int32_t *height,
              int32_t *rows_per_cta, int32_t *threads_wide, int32_t *threads_tall);
const char *ll_last_error(const ll_ctx *ctx); /* text of the last failure   */
/* Which passes run compile-time specialised kernels: bit 0 the wide (row)
 * pass, bit 1 the tall (column) pass (the others use the generic kernels);
 * bit 2: plain iterations run as fused cooperative launches; bit 3: every
 * step runs as cluster-resident launches (the state in the shared memory of
 * one thread-block cluster). */
int32_t ll_kernel_kinds(const ll_ctx *ctx);
/* Host-only self-check of the compiled kernel tables: the number of
 * specialised kernels whose stage-twiddle table (built on the host from the
 * recorded radix list) does not have the size the kernel reads, plus the
 * built-in launch preferences that do not give a specialised shape of their
 * width.  0 when consistent; needs no GPU. */
int32_t ll_check_tables(void);
const char *ll_status_string(ll_status s);

/* Test hook (CUDALucas.cu:2938-2950 handles a CUDA error from lucas_square
 * by resetting and restarting from the last checkpoint): the next `count`
 * ll_step calls return LL_ERR_INJECTED without touching the device. */
void ll_debug_inject_failure(ll_ctx *ctx, int32_t count);

/* Launches only the tall pass (square) or only the wide pass (carry) of one
 * iteration; used to time and profile the passes separately. */
ll_status ll_debug_launch(ll_ctx *ctx, int32_t which);

/* Batched mode (no counterpart in the reference, which tests one exponent per
 * process): `count` exponents q[i] at lengths n[i] advance together.  Each
 * member is a full context (ll_batch_member gives it for ll_load_digits,
 * ll_read_digits, ...); one step of `graph_iters` iterations of all members is
 * replayed from a single CUDA graph in which every member is a parallel
 * branch, so members of different lengths overlap on the GPU.  A member runs
 * exactly the kernels of a solo run: its residues equal the solo residues. */
typedef struct ll_batch ll_batch;
ll_status ll_batch_create(int device, int32_t count, const uint32_t *q, const uint32_t *n, int32_t graph_iters,
                          ll_batch **out);
void ll_batch_destroy(ll_batch *b);
int32_t ll_batch_size(const ll_batch *b);
ll_ctx *ll_batch_member(ll_batch *b, int32_t i);
ll_status ll_batch_start(ll_batch *b, const uint32_t *offsets);
/* iters iterations of every member; flags as ll_step (applied to each
 * member's last iteration); max_err[i] per member when a flag is given. */
ll_status ll_batch_step(ll_batch *b, uint32_t iters, uint32_t flags, float *max_err);
ll_status ll_batch_sync(ll_batch *b);
void *ll_batch_stream(const ll_batch *b);  /* stream the step graphs run on */
/* Members of one FFT length whose passes have specialised kernels form a
 * length class.  on = 1 (the default) makes one launch per pass run the pass
 * for every member of the class (the step graph then has one branch per
 * class, 2 kernel nodes per iteration); on = 0 launches every member's
 * passes separately (one branch per member).  On the 256-exponent
 * benchmark set the two measured 143.6 K and 141.2 K iterations/s.  Call
 * before the first ll_batch_step.  ll_batch_classes gives the number of
 * length classes. */
ll_status ll_batch_group_by_length(ll_batch *b, int32_t on);
int32_t ll_batch_classes(const ll_batch *b);
ll_status ll_batch_res64(ll_batch *b, uint64_t *res64);

/* Allocation-free LL steps.  No counterpart in the reference: CUDALucas
 * allocates its buffers with cudaMalloc in alloc_gpu_mem.  This entry point is
 * for callers that cannot allocate device memory -- code running inside an
 * arena or pool that owns all device memory, plugins whose host forbids
 * allocation during a work call, loops that must not touch the allocator.
 * It reads n balanced digits of x = s*2^offset from DEVICE memory digits_in,
 * runs `iters` LL iterations and writes the digits of the result (whose
 * offset is offset*2^iters mod q) to DEVICE memory digits_out; the max
 * roundoff error goes to the HOST float *max_err (may be NULL), as 1.0 when a
 * word left the exact FP64 range (the digits are then invalid).  All scratch
 * lives in one static array of LL_STATIC_SCRATCH_BYTES per device (held by
 * every GPU that loads the library, until exit); n may not exceed
 * LL_STATIC_MAX_WORDS (LL_ERR_ARG otherwise).  The first call on a device
 * looks up the array's device address; make that call before any stream
 * capture.  Calls share the array and it keeps the last call's contents:
 * calls whose GPU work overlapped would race.  Each call therefore holds a
 * lock of its device until its work has finished: it synchronises `stream`
 * (a cudaStream_t, NULL = legacy default stream) before it returns, also on
 * an error, and calls on different devices do not wait for each other. */
#define LL_STATIC_MAX_WORDS (1u << 20)
#define LL_STATIC_SCRATCH_BYTES (16u << 20)
ll_status ll_step_static(int device, uint32_t q, uint32_t n, uint32_t offset, uint32_t iters,
                         const int32_t *digits_in, int32_t *digits_out, float *max_err, void *stream);

/* ------------------------------------------------------------------------
 * Host helpers (no GPU needed).  Word j of an n-word representation of
 * 2^q-1 has floor(q/n)+1 bits iff ((-j*(q mod n)) mod n) < (q mod n).
 * ---------------------------------------------------------------------- */

/* Res64 of x*2^-offset mod 2^q-1 from any digit vector (exact; the digits
 * need not be balanced).  Same value as find_residue, CUDALucas.cu:1491. */
uint64_t ll_digits_res64(const int32_t *digits, uint32_t q, uint32_t n, uint32_t offset);

/* Canonicalises digits in place to 0 <= d_j < 2^bits_j with value in
 * [0, 2^q-1); returns 1 if the value is 0 mod 2^q-1 (standardize_digits,
 * CUDALucas.cu:1465). */
int32_t ll_digits_standardize(int32_t *digits, uint32_t q, uint32_t n);

/* pack_bits / unpack_bits / balance_digits, CUDALucas.cu:1594, :1285, :1313.
 * packed has (q+31)/32 words. */
void ll_pack_bits(const int32_t *digits, uint32_t *packed, uint32_t q, uint32_t n);
void ll_unpack_bits(const uint32_t *packed, int32_t *digits, uint32_t q, uint32_t n);
void ll_balance_digits(int32_t *digits, uint32_t q, uint32_t n);

/* checkpoint_checksum (CRC-32 style, poly 0x04C11DB7, CUDALucas.cu:1712) and
 * the additive ch_sum (CUDALucas.cu:1735). */
uint32_t ll_checkpoint_checksum(const void *bytes, size_t len);
uint32_t ll_additive_checksum(const uint32_t *words, size_t count);

/* FFT-length policy of CUDALucas (init_ffts / choose_fft_length,
 * CUDALucas.cu:947-1068) with the built-in 7-smooth table.
 * ll_fft_bounds gives the exponent's [lb, ub] word-count bounds;
 * ll_choose_fft_length returns the smallest table length >= max(lb, want)
 * that the engine supports and that is <= ub, or 0 if none. */
void ll_fft_bounds(uint32_t q, uint32_t *lb, uint32_t *ub);
uint32_t ll_choose_fft_length(uint32_t q, uint32_t want);
int32_t ll_fft_table(uint32_t *lengths, int32_t max_count);
int32_t ll_length_supported(uint32_t n);

/* init_ffts (CUDALucas.cu:947-1022) with a `<gpu> fft.txt` present: installs,
 * process-wide, the table made of the built-in lengths below the smallest
 * measured length, the measured lengths, and the built-in lengths above the
 * largest one, so that ll_choose_fft_length and ll_fft_table skip lengths the
 * benchmark found slower than a longer length.  `measured` is ascending (the
 * benchmark's list, in words); count 0 restores the built-in table.  Returns
 * the new table's size, -1 on a bad argument. */
int32_t ll_fft_table_merge(const uint32_t *measured, int32_t count);

/* The pruning rule of -cufftbench (CUDALucas.cu:2500-2513) over lengths in
 * ascending order with their measured ms/iter: keep[i] = 1 when length i is
 * faster than every longer length, or is a power of two in K.  Returns the
 * number kept, -1 on a bad argument. */
int32_t ll_fft_prune(const uint32_t *lengths, const float *ms_per_iter, int32_t count, int32_t *keep);

/* The largest exponent whose lower length bound (ll_fft_bounds) is <= n:
 * the `max exp` column of `<gpu> fft.txt`. */
uint32_t ll_fft_max_exponent(uint32_t n);

/* Name of CUDA device `device` (for the per-GPU `<gpu> fft.txt` and
 * `<gpu> shapes.txt` files); returns 0 on success. */
int32_t ll_device_name(int device, char *name, size_t len);

#ifdef __cplusplus
}
#endif
#endif /* LLB200_H */
