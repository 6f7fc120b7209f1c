// llucas: command-line Lucas-Lehmer tester on the B200 engine (libllb200).
//
// The host side of CUDALucas v2.06 re-built over the C ABI: the same flags
// (parse_args, CUDALucas.cu:3581-3818), ini keys (process_options,
// CUDALucas.cu:3388-3522), worktodo grammar (parse_worktodo_line,
// parse.c:241-471), checkpoint files c<q>/t<q>/s<q>.<iter>.<res64>
// (CUDALucas.cu:1746-1861), results lines (CUDALucas.cu:1581-1592,
// :3146-3178), self-test tables (-r, CUDALucas.cu:2650-2805) and the
// roundoff-error policy of check() (CUDALucas.cu:2862-3186).  The squaring
// itself is ll_step on the GPU; nothing here touches CUDA directly.
#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "llb200.h"

static const char kProgram[] = "llucas (B200 engine) v0.1";

// ------------------------------------------------------------- settings --
struct Config {
  std::string ini = "CUDALucas.ini";
  std::string workfile = "worktodo.txt";
  std::string results = "results.txt";
  std::string folder = "savefiles";
  int device = 0;
  int device_info = 0;
  int error_iters = 100;    // ErrorIterations
  int report_iters = 10000; // ReportIterations
  int check_iters = 100000; // CheckpointIterations
  int save_all = 0;         // SaveAllCheckpoints
  int polite = 0, polite_value = 50;
  int error_reset = 85;
  int error_limit = 40;     // ErrorLimit (percent)
  int roundoff_test = 0;    // RoundoffTest
  int selftest = -1;        // -r
  uint32_t fft_len = 0;     // -f / FFTLength
  bool quiet_ini = false;
  // Fault-injection hook for the recovery tests: LLUCAS_INJECT_FAILURES=J:C
  // makes C ll_step calls fail on the host (ll_debug_inject_failure): the
  // first call at or after iteration J fails, and after each restart the
  // next such call fails again, C times in all per process.
  uint32_t inject_at = 0;
  int inject_count = 0;
};

static int g_inject_left = -1;  // -1: not yet armed from the Config

static bool shape_for(const Config &cfg, uint32_t n, ll_tuning &tu);

static volatile sig_atomic_t g_quit = 0;
static void on_signal(int) { g_quit = 1; }

// ini lookup: "key=value" lines (IniGetInt/IniGetStr, parse.c:683-770)
static bool ini_get(const std::string &file, const char *key, std::string &out) {
  FILE *f = fopen(file.c_str(), "r");
  if (!f) return false;
  char line[1024];
  bool found = false;
  const size_t kl = strlen(key);
  while (fgets(line, sizeof line, f)) {
    char *p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (*p == '#' || *p == ';') continue;
    if (strncasecmp(p, key, kl) == 0 && p[kl] == '=') {
      std::string v = p + kl + 1;
      while (!v.empty() && (v.back() == '\n' || v.back() == '\r' || v.back() == ' ')) v.pop_back();
      out = v;
      found = true;
      break;
    }
  }
  fclose(f);
  return found;
}

static void ini_int(const Config &c, const char *key, int &v) {
  std::string s;
  if (ini_get(c.ini, key, s)) v = atoi(s.c_str());
}

// check_interval (CUDALucas.cu:3374): intervals are forced to k*10^m
static int check_interval(int v) {
  if (v <= 0) return 100;
  int m = 1;
  while (v / m >= 10) m *= 10;
  return (v / m) * m;
}

static uint32_t fft_from_str(const char *s) {
  char *end = nullptr;
  unsigned long v = strtoul(s, &end, 10);
  if (end && (*end == 'k' || *end == 'K')) v *= 1024;
  else if (end && (*end == 'm' || *end == 'M')) v *= 1024 * 1024;
  return (uint32_t)v;
}

static bool is_prime(uint32_t n) {
  if (n < 2) return false;
  if (n % 2 == 0) return n == 2;
  for (uint32_t i = 3; (uint64_t)i * i <= n; i += 2)
    if (n % i == 0) return false;
  return true;
}

// ------------------------------------------------------------ worktodo --
struct Assignment {
  uint32_t exponent = 0;
  uint32_t fft = 0;
  std::string key;
};

// One line of worktodo.txt: Test=[AID,]p[,nnnK] or DoubleCheck=...
// (parse_worktodo_line, parse.c:241-471).  Returns 1 for an assignment,
// 0 for a blank/comment line, -1 for a malformed line.
static int parse_line(const std::string &raw, Assignment &a) {
  std::string s = raw;
  while (!s.empty() && (s.back() == '\n' || s.back() == '\r')) s.pop_back();
  size_t i = 0;
  while (i < s.size() && isspace((unsigned char)s[i])) ++i;
  if (i == s.size()) return 0;
  if (s.compare(i, 2, "//") == 0 || s.compare(i, 2, "\\\\") == 0 || s[i] == '#') return 0;
  size_t eq;
  if (strncasecmp(s.c_str() + i, "Test=", 5) == 0) eq = i + 5;
  else if (strncasecmp(s.c_str() + i, "DoubleCheck=", 12) == 0) eq = i + 12;
  else return -1;
  std::string body = s.substr(eq);
  // strip a trailing comment
  for (const char *d : {"#", "//", "\\\\"}) {
    size_t c = body.find(d);
    if (c != std::string::npos) body = body.substr(0, c);
  }
  std::vector<std::string> f;
  size_t st = 0;
  while (true) {
    size_t c = body.find(',', st);
    std::string t = body.substr(st, c == std::string::npos ? std::string::npos : c - st);
    size_t a0 = t.find_first_not_of(" \t"), a1 = t.find_last_not_of(" \t");
    f.push_back(a0 == std::string::npos ? "" : t.substr(a0, a1 - a0 + 1));
    if (c == std::string::npos) break;
    st = c + 1;
  }
  size_t k = 0;
  a = Assignment();
  if (f.size() >= 2) {
    // first field is an assignment key when it is not a plain number
    bool numeric = !f[0].empty() && f[0].find_first_not_of("0123456789") == std::string::npos;
    if (!numeric) a.key = f[k++];
  }
  if (k >= f.size() || f[k].empty() || f[k].find_first_not_of("0123456789") != std::string::npos) return -1;
  a.exponent = (uint32_t)strtoul(f[k].c_str(), nullptr, 10);
  ++k;
  if (k < f.size() && !f[k].empty()) {
    const std::string &t = f[k];
    if (t.find_first_not_of("0123456789kKmM") != std::string::npos) return -1;
    a.fft = fft_from_str(t.c_str());
  }
  return 1;
}

// valid_assignment (parse.c:176-206)
static int valid_assignment(uint32_t exp, uint32_t fft) {
  if (exp < 7500) { fprintf(stderr, "Warning: exponents < 7500 are not supported!\n"); return 0; }
  if (fft % 1024) { fprintf(stderr, "Warning: FFT length %u is invalid, it must be a multiple of 1024.\n", fft); return 0; }
  if (!is_prime(exp)) { fprintf(stderr, "Warning: exponent is not prime!\n"); return -1; }
  return 1;
}

static bool next_assignment(const std::string &file, Assignment &out) {
  FILE *f = fopen(file.c_str(), "r");
  if (!f) { fprintf(stderr, "Can't open workfile %s\n\n", file.c_str()); return false; }
  char buf[1024];
  unsigned lineno = 0;
  bool ok = false;
  while (fgets(buf, sizeof buf, f)) {
    ++lineno;
    Assignment a;
    int r = parse_line(buf, a);
    if (r == 0) continue;
    if (r > 0 && valid_assignment(a.exponent, a.fft) > 0) { out = a; ok = true; break; }
    std::string l = buf;
    while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
    fprintf(stderr, "Warning: ignoring line %u: \"%s\" in \"%s\".\n", lineno, l.c_str(), file.c_str());
  }
  fclose(f);
  if (!ok) fprintf(stderr, "No valid assignment found.\n\n");
  return ok;
}

// clear_assignment (parse.c:572-678): drop the first line with this exponent
static bool clear_assignment(const std::string &file, uint32_t exponent) {
  FILE *f = fopen(file.c_str(), "r");
  if (!f) return false;
  std::vector<std::string> lines;
  char buf[1024];
  while (fgets(buf, sizeof buf, f)) lines.push_back(buf);
  fclose(f);
  std::string tmp = "__worktodo__.tmp";
  FILE *o = fopen(tmp.c_str(), "w");
  if (!o) return false;
  bool dropped = false;
  for (auto &l : lines) {
    Assignment a;
    if (!dropped && parse_line(l, a) > 0 && a.exponent == exponent) { dropped = true; continue; }
    fputs(l.c_str(), o);
  }
  fclose(o);
  return rename(tmp.c_str(), file.c_str()) == 0 && dropped;
}

// Appends under a <file>.lck lock file (fopen_and_lock, parse.c:775-894).
static bool append_locked(const std::string &file, const std::string &text) {
  std::string lck = file + ".lck";
  int fd = -1;
  for (int tries = 0; tries < 300; ++tries) {
    fd = open(lck.c_str(), O_CREAT | O_EXCL | O_WRONLY, 0644);
    if (fd >= 0 || errno != EEXIST) break;
    usleep(100000);
  }
  FILE *f = fopen(file.c_str(), "a");
  bool ok = f != nullptr;
  if (f) { fputs(text.c_str(), f); fclose(f); }
  if (fd >= 0) { close(fd); unlink(lck.c_str()); }
  return ok;
}

// ---------------------------------------------------------- checkpoints --
// Payload: (q+31)/32 words of the standardized residue (pack_bits of the
// digits, not de-rotated), then q, n, next iteration, offset, total time>>15,
// time adjustment>>15, iteration adjustment, 0, magic 0, CRC
// (set_checkpoint_data / write_checkpoint, CUDALucas.cu:1616-1625, :1798-1850).
struct Checkpoint {
  std::vector<uint32_t> words;  // end + 10 words
  uint32_t end = 0;
  bool valid = false;
};

static bool read_ck_file(const std::string &name, uint32_t q, Checkpoint &ck, bool backup) {
  FILE *f = fopen(name.c_str(), "rb");
  if (!f) return false;
  ck.end = (q + 31) / 32;
  ck.words.assign(ck.end + 10, 0);
  size_t got = fread(ck.words.data(), 4, ck.words.size(), f);
  fclose(f);
  // messages of read_checkpoint, CUDALucas.cu:1765-1792
  const char *bad = backup ? "\nThe backup appears to be corrupt. Restarting test.\n"
                           : "\nThe checkpoint appears to be corrupt. Trying the backup file.\n";
  if (got != ck.words.size()) {
    fputs(bad, stderr);
    return false;
  }
  const uint32_t stored = ck.words[ck.end + 9];
  const uint32_t crc = ll_checkpoint_checksum(ck.words.data(), 4 * (size_t)(ck.end + 9));
  // The reference writes every file with the CRC but checks the backup with
  // the additive ch_sum (CUDALucas.cu:1791 vs :1816), so backups never
  // validate there; here either checksum is accepted for the backup.
  bool ok = stored == crc || (backup && stored == ll_additive_checksum(ck.words.data(), ck.end + 9));
  if (!ok || ck.words[ck.end] != q) {
    fputs(bad, stderr);
    return false;
  }
  ck.valid = true;
  return true;
}

static Checkpoint read_checkpoint(uint32_t q) {
  Checkpoint ck;
  char c[64], t[64];
  snprintf(c, sizeof c, "c%u", q);
  snprintf(t, sizeof t, "t%u", q);
  if (read_ck_file(c, q, ck, false)) return ck;
  if (read_ck_file(t, q, ck, true)) return ck;
  ck = Checkpoint();
  return ck;
}

static void write_checkpoint(const Config &cfg, uint32_t q, std::vector<uint32_t> &w, uint64_t res) {
  const uint32_t end = (q + 31) / 32;
  char c[64], t[64];
  snprintf(c, sizeof c, "c%u", q);
  snprintf(t, sizeof t, "t%u", q);
  unlink(t);
  rename(c, t);
  w[end + 8] = 0;
  w[end + 9] = ll_checkpoint_checksum(w.data(), 4 * (size_t)(end + 9));
  FILE *f = fopen(c, "wb");
  if (!f) { fprintf(stderr, "Couldn't write checkpoint.\n"); return; }
  fwrite(w.data(), 4, end + 10, f);
  fclose(f);
  if (cfg.save_all > 0) {
    mkdir(cfg.folder.c_str(), 0755);
    char s[512];
    snprintf(s, sizeof s, "%s/s%u.%u.%016llx", cfg.folder.c_str(), q, w[end + 2] - 1, (unsigned long long)res);
    FILE *g = fopen(s, "wb");
    if (g) { fwrite(w.data(), 4, end + 10, g); fclose(g); }
  }
}

static void rm_checkpoint(uint32_t q) {
  char c[64], t[64];
  snprintf(c, sizeof c, "c%u", q);
  snprintf(t, sizeof t, "t%u", q);
  unlink(c);
  unlink(t);
}

// ---------------------------------------------------------------- output --
static std::string fmt_time(unsigned sec) {
  char b[64];
  unsigned d = sec / 86400, h = sec % 86400 / 3600, m = sec % 3600 / 60, s = sec % 60;
  if (d) snprintf(b, sizeof b, "%u:%02u:%02u:%02u", d, h, m, s);
  else if (h) snprintf(b, sizeof b, "%u:%02u:%02u", h, m, s);
  else snprintf(b, sizeof b, "%u:%02u", m, s);
  return b;
}

static double now_s() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}

// ------------------------------------------------------------------ test --
struct Run {
  ll_ctx *ctx = nullptr;
  uint32_t q = 0, n = 0;
  ~Run() { if (ctx) ll_destroy(ctx); }
};

static bool fail(ll_ctx *ctx, ll_status s, const char *what) {
  fprintf(stderr, "%s: %s%s%s\n", what, ll_status_string(s), ctx ? ": " : "", ctx ? ll_last_error(ctx) : "");
  return false;
}

// Next larger table length (g_fftlen++ in the reference's error policy).
static uint32_t next_length(uint32_t q, uint32_t n) {
  uint32_t lb, ub;
  ll_fft_bounds(q, &lb, &ub);
  std::vector<uint32_t> t(256);
  int cnt = ll_fft_table(t.data(), (int)t.size());
  for (int i = 0; i < cnt; ++i)
    if (t[i] > n && t[i] <= ub && ll_length_supported(t[i])) return t[i];
  return 0;
}

// check(q): one LL test with checkpoints, reports and the roundoff policy
// (CUDALucas.cu:2862-3186).  Returns 0 on completion, 1 when interrupted,
// 2 on an unrecoverable error.
// round_off_test (CUDALucas.cu:2589-2648): 1000 iterations with the error
// read back after every one.  Returns 1 when the average error exceeds 0.25
// or one iteration exceeds 0.35 (the caller moves to a longer FFT), 0 when
// the test may continue from the state reached (j and offset advanced, the
// last iteration reported), -1 on an engine error.
static int round_off_test(ll_ctx *c, uint32_t q, uint32_t n, uint32_t &j, uint32_t &offset) {
  printf("Running careful round off test for 1000 iterations.\n");
  printf("If average error > 0.25, or maximum error > 0.35,\n");
  printf("the test will restart with a longer FFT.\n");
  fflush(stdout);
  const uint32_t last = q - 2;
  float total = 0.f, max_err = 0.f, max_err1 = 0.f;
  uint32_t k = 0;
  const uint32_t count = last >= j ? std::min<uint32_t>(1000, last - j + 1) : 0;
  for (; k < count; ++k) {
    float e = 0.f;
    const ll_status s = ll_step(c, 1, k + 1 == count ? LL_REPORT : LL_ERRCHK, &e);
    if (s != LL_OK) { fail(c, s, "ll_step"); return -1; }
    if (e > max_err) max_err = e;
    if (e > max_err1) max_err1 = e;
    total += e;
    if (e > 0.35f) {
      printf("Iteration = %u < 1000 && err = %5.5f > 0.35, increasing n from %uK\n", k, e, n / 1024);
      return 1;
    }
    if (k && k % 100 == 0) {
      printf("Iteration  %u, average error = %5.5f, max error = %5.5f\n", k, total / k, max_err);
      max_err = 0.f;
    }
  }
  const float avg = total / 1000.0f;
  if (avg > 0.25f) {
    printf("Iteration 1000, average error = %5.5f > 0.25 (max error = %5.5f), increasing FFT length and "
           "restarting\n", avg, max_err);
    return 1;
  }
  printf("Iteration 1000, average error = %5.5f <= 0.25 (max error = %5.5f), continuing test.\n", avg, max_err1);
  offset = ll_offset(c);
  j += k;
  return 0;
}

// Applies the LLUCAS_INJECT_FAILURES hook: one failing ll_step call each
// time the test reaches iteration J, until C calls have failed.
static void maybe_inject(const Config &cfg, ll_ctx *c, uint32_t j) {
  if (g_inject_left < 0) g_inject_left = cfg.inject_count;
  if (g_inject_left > 0 && j >= cfg.inject_at) {
    ll_debug_inject_failure(c, 1);
    --g_inject_left;
  }
}

static int check(const Config &cfg, uint32_t q, uint32_t fft_req, const std::string &aid) {
  const uint32_t end = (q + 31) / 32;
  const uint32_t last = q - 2;
  const float error_limit = (float)((cfg.error_limit - cfg.error_limit / 8.0 * log((double)cfg.error_iters) / log(100.0)) / 100.0);
  Checkpoint ck = read_checkpoint(q);
  std::vector<uint32_t> state(end + 10, 0);   // last good state (packed + trailer)
  uint32_t j = 1, offset = 0, n0 = fft_req;
  bool fresh = true;
  if (ck.valid) {
    state = ck.words;
    j = state[end + 2];
    offset = state[end + 3];
    if (!n0) n0 = state[end + 1];
    fresh = false;
  } else {
    srand((unsigned)time(nullptr));
    offset = (uint32_t)(rand() % q);
  }
  uint32_t n = ll_choose_fft_length(q, n0 ? n0 : cfg.fft_len);
  if (!n) { fprintf(stderr, "No usable FFT length for exponent %u\n", q); return 2; }
  const uint32_t n_base = n;
  int retry = 1, fft_reset = 0;
  double total_time = fresh ? 0.0 : (double)((uint64_t)state[end + 4] << 15) * 1e-6;
  float maxerr_total = 0.f;
  std::vector<int32_t> digits;
  uint64_t res = 0;
  signal(SIGINT, on_signal);
  signal(SIGTERM, on_signal);

  while (true) {
    Run r;
    r.q = q;
    r.n = n;
    ll_tuning tu{};
    ll_status s = ll_create(cfg.device, q, n, shape_for(cfg, n, tu) ? &tu : nullptr, &r.ctx);
    if (s != LL_OK) { fail(nullptr, s, "ll_create"); return 2; }
    digits.assign(n, 0);
    if (fresh) {
      s = ll_start(r.ctx, offset);
      printf("Starting M%u fft length = %uK\n", q, n / 1024);
    } else {
      ll_unpack_bits(state.data(), digits.data(), q, n);
      ll_balance_digits(digits.data(), q, n);
      s = ll_load_digits(r.ctx, digits.data(), offset);
      printf("\nContinuing M%u @ iteration %u with fft length %uK, %5.2f%% done\n\n", q, j, n / 1024,
             100.0 * j / q);
    }
    if (s != LL_OK) { fail(r.ctx, s, "start"); return 2; }
    fflush(stdout);
    if (fresh && j == 1 && cfg.roundoff_test) {
      const int rt = round_off_test(r.ctx, q, n, j, offset);
      if (rt < 0) return 2;
      if (rt > 0) {
        const uint32_t nn = next_length(q, n);
        if (!nn) { printf("Something is wrong! Quitting.\n\n"); return 2; }
        n = nn;
        continue;  // a fresh start at the longer length
      }
      // the state after the round-off test is the first restart point
      s = ll_read_digits(r.ctx, digits.data(), &offset);
      if (s != LL_OK) { fail(r.ctx, s, "ll_read_digits"); return 2; }
      std::vector<int32_t> std_d(digits);
      ll_digits_standardize(std_d.data(), q, n);
      ll_pack_bits(std_d.data(), state.data(), q, n);
      state[end] = q;
      state[end + 1] = n;
      state[end + 2] = j;
      state[end + 3] = offset;
      fresh = false;
    }
    uint32_t last_report = j - 1;
    double t0 = now_s();
    float maxerr = 0.f;
    bool restart = false;
    // error read-back every 100 iterations (CUDALucas.cu:2936), or every
    // PoliteValue iterations in polite mode (CUDALucas.cu:1979)
    const uint32_t chunk = cfg.polite && cfg.polite_value > 0 && cfg.polite_value < 100 ? cfg.polite_value : 100;
    while (j <= last) {
      // advance to the next multiple of the chunk, report or checkpoint boundary
      uint32_t stop = (j / chunk + 1) * chunk;
      const uint32_t rep = (j / cfg.report_iters + 1) * cfg.report_iters;
      if (rep < stop) stop = rep;
      if (stop > last) stop = last;
      if (stop < j) stop = j;
      const bool report = (stop % cfg.report_iters == 0) || stop == last || g_quit;
      float err = 0.f;
      maybe_inject(cfg, r.ctx, j);
      s = ll_step(r.ctx, stop - j + 1, report ? LL_REPORT : LL_ERRCHK, &err);
      if (s != LL_OK) {
        fail(r.ctx, s, "ll_step");
        printf("Resetting device and restarting from last checkpoint.\n\n");
        restart = true;
        break;
      }
      offset = ll_offset(r.ctx);
      j = stop;
      if (err > maxerr) maxerr = err;
      if (err > error_limit) {
        printf("Round off error at iteration = %u, err = %0.5g > %0.5g, fft = %uK.\n", j, err, error_limit, n / 1024);
        if (retry) {
          printf("Restarting from last checkpoint to see if the error is repeatable.\n\n");
          retry = 0;
        } else if (fft_reset) {
          printf("The error won't go away. I give up.\n\n");
          return 2;
        } else {
          uint32_t nn = next_length(q, n);
          if (!nn) { printf("Something is wrong! Quitting.\n\n"); return 2; }
          printf("The error persists.\nTrying a larger fft until the next checkpoint.\n\n");
          n = nn;
          fft_reset = 1;
        }
        restart = true;
        break;
      }
      if (report) {
        s = ll_read_digits(r.ctx, digits.data(), &offset);
        if (s != LL_OK) { fail(r.ctx, s, "ll_read_digits"); return 2; }
        res = ll_digits_res64(digits.data(), q, n, offset);
        const double t1 = now_s();
        const double dt = t1 - t0;
        total_time += dt;
        t0 = t1;
        const double ms = dt * 1000.0 / (double)(j - last_report);
        last_report = j;
        if (j < last) {
          const unsigned eta = (unsigned)(ms * (last - j) / 1000.0);
          printf("Iteration %u / %u, 0x%016llx, %uK, %s, error = %5.5f, real: %s, %4.4f ms/iter, ETA: %s, %5.2f%%\n",
                 j, q, (unsigned long long)res, n / 1024, kProgram, maxerr, fmt_time((unsigned)dt).c_str(), ms,
                 fmt_time(eta).c_str(), 100.0 * j / q);
          fflush(stdout);
          if (res == 0 || res == 2) {
            printf("Illegal residue: 0x%016llx. See mersenneforum.org for help.\n\n", (unsigned long long)res);
            return 2;
          }
        }
        // keep the state as the restart point (the reference repacks at each report)
        std::vector<int32_t> std_d(digits);
        ll_digits_standardize(std_d.data(), q, n);
        ll_pack_bits(std_d.data(), state.data(), q, n);
        state[end] = q;
        state[end + 1] = n;
        state[end + 2] = j + 1;
        state[end + 3] = offset;
        state[end + 4] = (uint32_t)((uint64_t)(total_time * 1e6) >> 15);
        if (maxerr > maxerr_total) maxerr_total = maxerr;
        if (j % cfg.check_iters == 0 || g_quit || j == last) write_checkpoint(cfg, q, state, res);
        if (fft_reset) {
          printf("Resettng fft.\n\n");
          n = n_base;
          fft_reset = 0;
          retry = 1;
          fresh = false;
          ++j;
          restart = true;
          break;
        } else if (!retry) {
          printf("Looks like the error went away, continuing.\n\n");
          retry = 1;
        }
        maxerr = maxerr * cfg.error_reset / 100.0f;
        if (g_quit) {
          printf(" Estimated time spent so far: %s\n\n", fmt_time((unsigned)total_time).c_str());
          return 1;
        }
      }
      ++j;
    }
    if (restart) {
      // resume from the last good packed state
      if (state[end + 2]) {
        j = state[end + 2];
        offset = state[end + 3];
        fresh = false;
      } else {
        j = 1;
        fresh = true;
      }
      continue;
    }
    break;
  }
  // final result (CUDALucas.cu:3146-3178)
  char line[512];
  if (res == 0) {
    printf("M( %u )P, n = %uK, %s", q, n / 1024, kProgram);
    snprintf(line, sizeof line, "M( %u )P, offset = %u, n = %uK, %s", q, offset, n / 1024, kProgram);
  } else {
    printf("M( %u )C, 0x%016llx, offset = %u, n = %uK, %s", q, (unsigned long long)res, offset, n / 1024, kProgram);
    snprintf(line, sizeof line, "M( %u )C, 0x%016llx, offset = %u, n = %uK, %s", q, (unsigned long long)res,
             offset, n / 1024, kProgram);
  }
  printf(", estimated total time = %s\n\n", fmt_time((unsigned)total_time).c_str());
  std::string out = line;
  if (!aid.empty() && strncasecmp(aid.c_str(), "N/A", 3) != 0) out += ", AID: " + aid;
  out += "\n";
  if (!append_locked(cfg.results, out)) fprintf(stderr, "Cannot write results to %s\n\n", cfg.results.c_str());
  if (res) rm_checkpoint(q);
  fflush(stdout);
  return 0;
}

// ------------------------------------------------------------- self-test --
// Res64 of s_10000 (s0 = 4) for the reference's self-test exponents: the
// short table (-r 0, CUDALucas.cu:2673-2682) and the long one (-r 1,
// CUDALucas.cu:2684-2729), kept as the known answers.
struct Kat { uint32_t p; uint64_t r; };
static const Kat kShort[] = {
    {86243, 0x23992ccd735a03d9ull},   {132049, 0x4c52a92b54635f9eull},  {216091, 0x30247786758b8792ull},
    {756839, 0x5d2cbe7cb24a109aull},  {859433, 0x3c4ad525c2d0aed0ull},  {1257787, 0x3f45bf9bea7213eaull},
    {1398269, 0xa4a6d2f0e34629dbull}, {2976221, 0x2a7111b7f70fea2full}, {3021377, 0x6387a70a85d46bafull},
    {6972593, 0x88f1d2640adb89e1ull}, {13466917, 0x9fdc1f4092b15d69ull}, {20996011, 0x5fc58920a821da11ull},
    {24036583, 0xcbdef38a0bdc4f00ull}, {25964951, 0x62eb3ff0a5f6237cull}, {30402457, 0x0b8600ef47e69d27ull},
    {32582657, 0x02751b7fcec76bb1ull}, {37156667, 0x67ad7646a1fad514ull}, {42643801, 0x8f90d78d5007bba7ull},
    {43112609, 0xe86891ebf6cd70c4ull}, {57885161, 0x76c27556683cd84dull}};
static const Kat kLong[] = {
    {22133, 0xb3ed67a5d4be2a9full}, {43633, 0xa3f3e669e061bfbeull}, {85933, 0x474e01b06d9698f8ull},
    {169409, 0x3d32414583ac7d9aull}, {190097, 0xf681a2a2ad0397fbull}, {210739, 0x7e3b5a8b4e4c43a0ull},
    {292921, 0xade86fd9a4ad99f1ull}, {333803, 0xe7311b6b953a609full}, {374587, 0xdb4ca1fad1c3e276ull},
    {435571, 0xb6711834a5dd0ad1ull}, {657719, 0xc56715170d6819efull}, {738083, 0x2d6f637091a3ce6dull},
    {818239, 0xe63f1cc63af264cbull}, {978041, 0xc049101d2a0f945bull}, {1137271, 0x8e006ecd6719158full},
    {1216693, 0x847bbf5d0a077cadull}, {1296011, 0xc5002ae321cc3055ull}, {1414741, 0x7c6237b4f067d8caull},
    {1612249, 0xfd4c832d1dbf746full}, {1927129, 0x155eb42707e90cd9ull}, {2240863, 0xf5e629fcc1247e4aull},
    {2397383, 0xf58df7be5d73b369ull}, {2553659, 0x0a9357c955a13ca5ull}, {2865601, 0xdac4555e41809026ull},
    {3176779, 0x1a8ed18fa285f151ull}, {3215629, 0x9e0c8eb95b15ae66ull}, {3332107, 0x7a539a9b8060b0d8ull},
    {3564823, 0x820e428ad972cd86ull}, {3797219, 0xa7223e4ecad04860ull}, {3874583, 0xf60c0a837ec80a50ull},
    {3951977, 0xb5da72b662eb3652ull}, {4415431, 0x31d58de3e1d79a85ull}, {4723783, 0x89fac94192cc3becull},
    {5031737, 0x6371a0f4aef2af32ull}, {5646379, 0xf03d3bbaa51fbe63ull}, {6259537, 0x026805e6b4f1b0feull},
    {6336103, 0x0f0718d2da4aaad3ull}, {6565633, 0x98d84929de4e6f63ull}, {7024163, 0xc030210791a14e9cull},
    {7482053, 0xf54842c06ba7e3c4ull}, {7634537, 0x24872a305faae4f8ull}, {7786967, 0x060dfca872385f9bull},
    {8700169, 0x4f95b9afd65b3c7eull}, {9914521, 0xc6ff39fd699d624cull}, {11125619, 0x1484b22a17312da0ull},
    {12333809, 0xbd8435b83f062d6aull}, {12484649, 0xd56aa903718b2353ull}, {12936919, 0x1527f970ad3020bfull},
    {13840423, 0x002a2aa0b97306b7ull}, {14742617, 0xf63addc70cde0addull}, {15043099, 0xe52f5e2045a2db30ull},
    {15343429, 0x5eda3ab1816505b9ull}, {16543493, 0x85ea99f94dc20a8bull}, {17142793, 0x94edb737270e4ca7ull},
    {17217653, 0x3ec0aa4728b97ef3ull}, {19535569, 0x708d03d1fe4c06f2ull}, {21921901, 0x38651890258c09bbull},
    {22368691, 0xcc264d5bc61bc957ull}, {24599717, 0x76e7ab92aca768abull}, {25490893, 0x135f7e63e7357efbull},
    {27271147, 0xb1a47be0366530efull}, {29640913, 0x4d51f44ffae1c913ull}, {30232693, 0xcab02c7178561218ull},
    {32597297, 0xec15163c817fcfddull}, {33778141, 0x9145db2f2080172eull}, {38492887, 0x36efe22824adb35cull},
    {43194913, 0xf13bdac634316fa2ull}, {47885689, 0x51a71b010cacfd92ull}, {48471289, 0x5f504f82abefdd1cull},
    {50227213, 0x643739d94fe6789cull}, {53735041, 0x653267115ab57688ull}, {58404433, 0x6e4b3224349080c8ull},
    {59570449, 0x8d7c6550107a2d0aull}, {64229677, 0x796701d5562dce22ull}, {66556463, 0xe418b5d4fb5c7e45ull},
    {66847171, 0xc01ffc681dbb8966ull}, {75846319, 0x626ab6b09b607ba9ull}, {85111207, 0x14bb68062d100ebdull},
    {86845813, 0x88220ac98093b65cull}, {95507747, 0xa92c24ad9b6655f1ull}, {97454309, 0xd6d4b3b14c1b73d8ull},
    {105879517, 0x3310a4b03a18f4a8ull}, {111056879, 0x59e95ddb73c59624ull}, {115080019, 0x293d0b202c9e3c63ull},
    {117377567, 0xdf57cd5d866f1065ull}, {118813021, 0x1cd6a8caef092277ull}, {126558077, 0x40b1cf42af7f99a7ull},
    {131142761, 0x046ab21b10a27189ull}, {131715607, 0x8fcfb36b868738ecull}, {142017539, 0x801794367f35ccb6ull},
    {147162241, 0x72c8773764a260b0ull}, {149447533, 0x24702427a0f5d673ull},
};

// check_residue (CUDALucas.cu:2731-2805): 10000 iterations of each table
// exponent at its default length, with the round-off test first when
// RoundoffTest is set; an iteration error above 0.4 moves to the next
// length and restarts the exponent.
static int selftest(const Config &cfg) {
  int bad = 0;
  const Kat *tab = cfg.selftest ? kLong : kShort;
  const size_t cnt = cfg.selftest ? sizeof(kLong) / sizeof(kLong[0]) : sizeof(kShort) / sizeof(kShort[0]);
  const uint32_t last = 10000;
  for (size_t t = 0; t < cnt; ++t) {
    const Kat &k = tab[t];
    uint32_t n = ll_choose_fft_length(k.p, 0);
    uint64_t r = 0;
    float maxerr = 0.f;
    double dt = 0.0;
    bool restarting;
    bool first = true;
    do {
      restarting = false;
      if (!n) { fprintf(stderr, "No usable FFT length for M%u\n", k.p); return 2; }
      ll_ctx *c = nullptr;
      ll_tuning tu{};
      ll_status s = ll_create(cfg.device, k.p, n, shape_for(cfg, n, tu) ? &tu : nullptr, &c);
      if (s != LL_OK) { fail(nullptr, s, "ll_create"); return 2; }
      if (first) printf("Starting self test M%u fft length = %uK\n", k.p, n / 1024);
      first = false;
      const double t0 = now_s();
      uint32_t j = 1, offset = (uint32_t)(rand() % k.p);
      s = ll_start(c, offset);
      if (s == LL_OK && cfg.roundoff_test) {
        const int rt = round_off_test(c, k.p, n, j, offset);
        if (rt < 0) { ll_destroy(c); return 2; }
        if (rt > 0) restarting = true;
      }
      maxerr = 0.f;
      while (s == LL_OK && !restarting && j <= last) {
        const uint32_t stop = std::min<uint32_t>((j / 100 + 1) * 100, last);
        float err = 0.f;
        s = ll_step(c, stop - j + 1, stop == last ? LL_REPORT : LL_ERRCHK, &err);
        if (err > maxerr) maxerr = err;
        if (err > 0.4f) restarting = true;
        j = stop + 1;
      }
      if (s == LL_OK && !restarting) s = ll_res64(c, &r);
      if (s != LL_OK) { fail(c, s, "self test"); ll_destroy(c); return 2; }
      ll_destroy(c);
      dt = now_s() - t0;
      if (restarting) n = next_length(k.p, n);
    } while (restarting);
    printf("Iteration %u / %u, 0x%016llx, %uK, %s, error = %5.5f, real: %s, %4.4f ms/iter\n", last, k.p,
           (unsigned long long)r, n / 1024, kProgram, maxerr, fmt_time((unsigned)dt).c_str(), dt * 1000.0 / last);
    if (r != k.r) {
      printf("Expected residue [%016llx] does not match actual residue [%016llx]\n\n", (unsigned long long)k.r,
             (unsigned long long)r);
      ++bad;
    } else
      printf("This residue is correct.\n\n");
    fflush(stdout);
  }
  if (bad) fprintf(stderr, "Error: There %s %d bad selftest%s!\n", bad > 1 ? "were" : "was", bad, bad > 1 ? "s" : "");
  return bad ? 1 : 0;
}

// ------------------------------------------------------------ fft.txt --
// `<gpu> fft.txt` in the reference's layout (CUDALucas.cu:2555-2573): device
// lines, a header, then one "%5d %10d %8.4f" row per kept length (length in
// K, largest exponent, ms/iter).  init_ffts reads every line whose leading
// number is non-zero as a length in K (CUDALucas.cu:975-990).
static std::vector<uint32_t> read_fft_file(const std::string &name) {
  std::vector<uint32_t> out;
  FILE *f = fopen(name.c_str(), "r");
  if (!f) return out;
  char buf[192];
  while (fgets(buf, sizeof buf, f)) {
    const int k = atoi(buf);
    if (k > 0) out.push_back((uint32_t)k * 1024u);
  }
  fclose(f);
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// -cufftbench s e passes (CUDALucas.cu:2413-2587): times every supported
// length from s K to e K (passes x 50 iterations after a warm-up of 50),
// keeps the lengths faster than every longer one (and the powers of two),
// writes them to `<gpu> fft.txt`, moving an older file aside as the
// reference does.  For each length the fastest launch choice among the
// engine's candidates (row width W; for the engine's own width also the
// kernel variants: two launches instead of the cluster-resident step, the
// alternative row kernel) goes to `<gpu> shapes.txt` as width and
// ll_tuning.kernels.
static int cufftbench(const Config &cfg, const char *gpu, int s, int e, int passes) {
  if (!gpu[0]) { fprintf(stderr, "no CUDA device %d\n", cfg.device); return 2; }
  std::vector<uint32_t> lens;
  std::vector<float> times;
  std::vector<int32_t> widths, kernels;
  for (int k = s; k <= e; ++k) {
    const uint32_t n = (uint32_t)k * 1024u;
    if (!ll_length_supported(n)) continue;
    uint32_t q = (uint32_t)(n * 17.6) | 1;
    while (!is_prime(q)) q += 2;
    float best = 0.f;
    int32_t best_w = 0, best_k = 0;
    // candidates: the engine's own choice, its kernel variants, then the
    // divisors of N = n/2 near its square root as row widths
    std::vector<std::pair<int32_t, int32_t>> cand = {{0, 0}, {0, LL_KERNELS_NO_CLUSTER}, {0, LL_KERNELS_ALT_WIDE}};
    const uint32_t N = n / 2;
    for (uint32_t w = 64; w <= 8192 && w <= N; w += 2)
      if (N % w == 0 && (double)w * w >= N / 16.0 && (double)w * w <= 16.0 * N) cand.push_back({(int32_t)w, 0});
    int32_t def_w = 0, def_tw = 0, def_kinds = -1;
    for (const auto &wk : cand) {
      const int32_t w = wk.first;
      ll_tuning tu{};
      tu.width = w;
      tu.kernels = wk.second;
      ll_ctx *c = nullptr;
      if (ll_create(cfg.device, q, n, (w || wk.second) ? &tu : nullptr, &c) != LL_OK) continue;
      int32_t W = 0, TW = 0;
      ll_shape(c, &W, nullptr, nullptr, &TW, nullptr);
      const int32_t kinds = ll_kernel_kinds(c);
      if (w && w != W) { ll_destroy(c); continue; }
      if (!w && !wk.second) { def_w = W; def_tw = TW; def_kinds = kinds; }
      // a variant that changes nothing, or the engine's width again, is not timed twice
      if ((!w && wk.second && W == def_w && TW == def_tw && kinds == def_kinds) || (w && w == def_w)) {
        ll_destroy(c);
        continue;
      }
      float err = 0.f;
      ll_start(c, 0);
      ll_step(c, 50, LL_ERRCHK, &err);
      const double t0 = now_s();
      const ll_status st = ll_step(c, 50 * (uint32_t)passes, LL_ERRCHK, &err);
      const float ms = (float)((now_s() - t0) * 1000.0 / (50.0 * passes));
      ll_destroy(c);
      if (st != LL_OK) continue;
      if (best == 0.f || ms < best) { best = ms; best_w = W; best_k = wk.second; }
    }
    if (best == 0.f) continue;
    printf("fft size = %uK, ave time = %6.4f msec, width %d, kernels %d\n", n / 1024, best, best_w, best_k);
    fflush(stdout);
    lens.push_back(n);
    times.push_back(best);
    widths.push_back(best_w);
    kernels.push_back(best_k);
  }
  std::vector<int32_t> keep(lens.size(), 0);
  ll_fft_prune(lens.data(), times.data(), (int32_t)lens.size(), keep.data());
  const std::string name = std::string(gpu) + " fft.txt";
  char stamp[64];
  const time_t now = time(nullptr);
  strftime(stamp, sizeof stamp, "%d%H%M%S", localtime(&now));
  const std::string bak = std::string(gpu) + " fft" + stamp + ".txt";
  unlink(bak.c_str());
  rename(name.c_str(), bak.c_str());
  FILE *f = fopen(name.c_str(), "w");
  FILE *g = fopen((std::string(gpu) + " shapes.txt").c_str(), "w");
  if (!f) { fprintf(stderr, "Cannot open %s.\n", name.c_str()); return 2; }
  fprintf(f, "Device              %s\n\n  fft    max exp  ms/iter\n", gpu);
  if (g) fprintf(g, "# fft(K) width ms/iter kernels\n");
  for (size_t i = 0; i < lens.size(); ++i) {
    if (g) fprintf(g, "%5u %6d %8.4f %d\n", lens[i] / 1024, widths[i], times[i], kernels[i]);
    if (keep[i]) fprintf(f, "%5u %10u %8.4f\n", lens[i] / 1024, ll_fft_max_exponent(lens[i]), times[i]);
  }
  fclose(f);
  if (g) fclose(g);
  printf("Old %s moved to %s.\nOptimal fft lengths saved in %s.\n", name.c_str(), bak.c_str(), name.c_str());
  return 0;
}

// The launch shape measured fastest for length n (`<gpu> shapes.txt`), if any.
static bool shape_for(const Config &cfg, uint32_t n, ll_tuning &tu) {
  char gpu[256];
  if (ll_device_name(cfg.device, gpu, sizeof gpu)) return false;
  FILE *f = fopen((std::string(gpu) + " shapes.txt").c_str(), "r");
  if (!f) return false;
  char buf[192];
  bool found = false;
  while (fgets(buf, sizeof buf, f)) {
    unsigned k = 0;
    int w = 0, kern = 0;
    float ms = 0.f;
    if (buf[0] != '#' && sscanf(buf, "%u %d %f %d", &k, &w, &ms, &kern) >= 2 && k * 1024u == n && w > 0) {
      tu = ll_tuning{};
      tu.width = w;
      tu.kernels = kern & (LL_KERNELS_NO_CLUSTER | LL_KERNELS_ALT_WIDE);  // the variants the table may choose
      found = true;
    }
  }
  fclose(f);
  return found;
}

// ------------------------------------------------------------------ main --
static void usage() {
  printf("%s\nUsage: llucas [-d device] [-i inifile] [-f fft] [-x report] [-c checkpoint] [-s folder]\n"
         "              [-e limit] [-polite n] [-r 0|1] [-cufftbench s e passes] [-v] [-h]\n"
         "              [exponent | worktodo file]\n", kProgram);
}

int main(int argc, char **argv) {
  Config cfg;
  // -i must be seen before the ini is read
  for (int i = 1; i + 1 < argc; ++i)
    if (!strcmp(argv[i], "-i")) cfg.ini = argv[i + 1];
  {
    std::string v;
    if (ini_get(cfg.ini, "WorkFile", v)) cfg.workfile = v;
    if (ini_get(cfg.ini, "ResultsFile", v)) cfg.results = v;
    if (ini_get(cfg.ini, "SaveFolder", v)) cfg.folder = v;
    if (ini_get(cfg.ini, "FFTLength", v)) cfg.fft_len = fft_from_str(v.c_str());
    ini_int(cfg, "DeviceNumber", cfg.device);
    ini_int(cfg, "PrintDeviceInfo", cfg.device_info);
    ini_int(cfg, "ErrorIterations", cfg.error_iters);
    ini_int(cfg, "ReportIterations", cfg.report_iters);
    ini_int(cfg, "CheckpointIterations", cfg.check_iters);
    ini_int(cfg, "SaveAllCheckpoints", cfg.save_all);
    ini_int(cfg, "Polite", cfg.polite);
    ini_int(cfg, "PoliteValue", cfg.polite_value);
    ini_int(cfg, "ErrorReset", cfg.error_reset);
    ini_int(cfg, "ErrorLimit", cfg.error_limit);
    ini_int(cfg, "RoundoffTest", cfg.roundoff_test);
  }
  std::string target;
  int bench_s = 0, bench_e = 0, bench_p = 0;
  for (int i = 1; i < argc; ++i) {
    const char *a = argv[i];
    auto need = [&](int k) {
      if (i + k >= argc) { fprintf(stderr, "can't parse %s option\n\n", a); exit(2); }
    };
    if (!strcmp(a, "-h")) { usage(); return 0; }
    else if (!strcmp(a, "-v")) { printf("%s\n\n", kProgram); return 0; }
    else if (!strcmp(a, "-d")) { need(1); cfg.device = atoi(argv[++i]); }
    else if (!strcmp(a, "-i")) { need(1); ++i; }
    else if (!strcmp(a, "-f")) { need(1); cfg.fft_len = fft_from_str(argv[++i]); }
    else if (!strcmp(a, "-x")) { need(1); cfg.report_iters = atoi(argv[++i]); }
    else if (!strcmp(a, "-c")) { need(1); cfg.check_iters = atoi(argv[++i]); }
    else if (!strcmp(a, "-s")) { need(1); cfg.save_all = 1; cfg.folder = argv[++i]; }
    else if (!strcmp(a, "-e")) { need(1); cfg.error_limit = atoi(argv[++i]); }
    else if (!strcmp(a, "-polite")) { need(1); cfg.polite = 1; cfg.polite_value = atoi(argv[++i]); }
    else if (!strcmp(a, "-r")) {
      cfg.selftest = 0;
      if (i + 1 < argc && argv[i + 1][0] != '-') cfg.selftest = atoi(argv[++i]);
    } else if (!strcmp(a, "-k") || !strcmp(a, "-info")) {
      /* interactive keys: not supported (no TTY handling); -info: shown below */
      if (!strcmp(a, "-info")) cfg.device_info = 1;
    } else if (!strcmp(a, "-threads")) { need(2); i += 2; /* shapes are chosen by the engine */ }
    else if (!strcmp(a, "-cufftbench")) {
      need(3);
      bench_s = atoi(argv[i + 1]);
      bench_e = atoi(argv[i + 2]);
      bench_p = atoi(argv[i + 3]);
      i += 3;
    } else if (!strcmp(a, "-worktodo-check")) {
      // parse a worktodo file and print the assignments (no GPU needed)
      need(1);
      FILE *f = fopen(argv[i + 1], "r");
      if (!f) { fprintf(stderr, "Can't open workfile %s\n", argv[i + 1]); return 1; }
      char buf[1024];
      while (fgets(buf, sizeof buf, f)) {
        Assignment as;
        int r = parse_line(buf, as);
        if (r > 0) printf("assignment exponent=%u fft=%u key=%s valid=%d\n", as.exponent, as.fft, as.key.c_str(),
                          valid_assignment(as.exponent, as.fft));
        else if (r < 0) printf("invalid\n");
      }
      fclose(f);
      return 0;
    } else if (!strcmp(a, "-memtest") || !strcmp(a, "-threadbench")) {
      fprintf(stderr, "%s is not provided by this engine (see -cufftbench for timings)\n", a);
      return 2;
    } else if (a[0] == '-') { fprintf(stderr, "unknown option %s\n", a); usage(); return 2; }
    else target = a;
  }
  cfg.report_iters = check_interval(cfg.report_iters);
  cfg.check_iters = check_interval(cfg.check_iters);
  if (const char *inj = getenv("LLUCAS_INJECT_FAILURES")) {
    unsigned at = 0;
    int cnt = 0;
    if (sscanf(inj, "%u:%d", &at, &cnt) == 2) {
      cfg.inject_at = at;
      cfg.inject_count = cnt;
    }
  }
  char gpu[256] = "";
  const bool have_gpu = ll_device_name(cfg.device, gpu, sizeof gpu) == 0;
  if (bench_p > 0) return cufftbench(cfg, gpu, bench_s, bench_e, bench_p);
  // init_ffts (CUDALucas.cu:975-1021): a `<gpu> fft.txt` written by an
  // earlier -cufftbench restricts the lengths inside its range to the
  // measured ones
  if (have_gpu) {
    const std::vector<uint32_t> measured = read_fft_file(std::string(gpu) + " fft.txt");
    if (!measured.empty()) ll_fft_table_merge(measured.data(), (int32_t)measured.size());
  }
  if (cfg.selftest >= 0) return selftest(cfg);
  if (target.empty()) target = cfg.workfile;
  char *endp = nullptr;
  unsigned long q = strtoul(target.c_str(), &endp, 10);
  if (endp && *endp == '\0' && q > 0) {
    if (valid_assignment((uint32_t)q, cfg.fft_len ? cfg.fft_len : 1024) <= 0) return 2;
    return check(cfg, (uint32_t)q, cfg.fft_len, "");
  }
  cfg.workfile = target;
  Assignment a;
  while (!g_quit && next_assignment(cfg.workfile, a)) {
    int r = check(cfg, a.exponent, a.fft ? a.fft : cfg.fft_len, a.key);
    if (r != 0) return r;
    clear_assignment(cfg.workfile, a.exponent);
  }
  return 0;
}
