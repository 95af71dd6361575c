/*
 * gnm_oracle.c — CPU oracle for gnomon's polygenic-score hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls this
 * file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it (through oracle/oracle.py), and only as the checker / timed CPU
 * baseline.
 *
 * The reference (SauersML/gnomon, Rust nightly) cannot be built here (no
 * cargo/rustc, crates not vendored), so this is a restatement in plain C of
 * its CPU scoring engine, following:
 *   score/prepare.rs:197-208      flip folding (dosage_weight, missing_correction)
 *   score/prepare.rs:644-646      baseline = sum of missing_correction (f64)
 *   score/decide.rs:69-250        run strategy + per-variant path trees
 *   score/batch.rs:583-614        popcnt density estimate used for routing
 *   score/batch.rs:622-844        variant-major ("NoPivot") path, f64 direct
 *   score/batch.rs:48-422         person-major ("Pivot") path: per person per
 *                                 <=256-variant mini-batch: missing first
 *                                 (count++, sum -= corr in f64), then f32
 *                                 accumulation over dosage-1 rows (ascending)
 *                                 then dosage-2 rows (fma(w,2,acc)), flushed
 *                                 to f64 (kernel.rs:34-301)
 *   score/pipeline.rs:1739-1775   output initialised to the baseline
 *   score/pipeline.rs:766-795     final = baseline + sparse partial + dense partial
 *   score/pipeline.rs:1921-2049   dense rows batched 256 at a time
 * plus an independent extended-precision per-genotype scorer used as the
 * "FP64 oracle" for error reports, and the synthetic genotype generator that
 * the CUDA generator must reproduce bit for bit.
 *
 * Parity of this restatement is pinned by the reference's own known-answer
 * tests (batch.rs:1013-1114, prepare.rs:1041-1097) reproduced in
 * tests/golden/ and by an independent numpy decoder.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Synthetic generator (shared definition with the CUDA generator)          */
/* ------------------------------------------------------------------------ */

/* SplitMix64 finaliser (Steele, Lea, Flood 2014). */
static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static inline uint64_t synth_key(uint64_t seed, uint64_t v, uint64_t i) {
  return mix64(seed) ^ (v * 0xD1B54A32D192ED03ull) ^ (i * 0x8CB92BA72F3D8DD7ull);
}

static inline uint32_t synth_code(uint64_t seed, uint64_t v, uint64_t i, const uint32_t* thr) {
  uint64_t x = mix64(synth_key(seed, v, i));
  uint32_t um = (uint32_t)x, ug = (uint32_t)(x >> 32);
  if (um < thr[0]) return 1u;
  if (ug < thr[1]) return 0u;
  if (ug < thr[2]) return 2u;
  return 3u;
}

/* rows: variant v (absolute index variant_begin+j) at rows + j*pitch.
 * thr: [num_variants][3] thresholds for variants variant_begin.. */
void oracle_synth_rows(uint8_t* rows, uint64_t pitch, uint64_t variant_begin,
                       uint64_t num_variants, uint64_t num_people,
                       const uint32_t* thr, uint64_t seed) {
  uint64_t bpv = (num_people + 3) / 4;
  for (uint64_t j = 0; j < num_variants; ++j) {
    uint8_t* row = rows + j * pitch;
    const uint32_t* t = thr + 3 * j;
    uint64_t v = variant_begin + j;
    for (uint64_t b = 0; b < bpv; ++b) {
      uint8_t byte = 0;
      for (uint64_t q = 0; q < 4; ++q) {
        uint64_t i = 4 * b + q;
        if (i < num_people) byte |= (uint8_t)(synth_code(seed, v, i, t) << (2 * q));
      }
      row[b] = byte;
    }
    for (uint64_t b = bpv; b < pitch; ++b) row[b] = 0;
  }
}

/* Decode to {0,1,2} and -1 for missing (batch.rs:489-503 semantics). */
void oracle_decode(const uint8_t* rows, uint64_t pitch, uint64_t num_variants,
                   uint64_t num_people, int8_t* out, uint64_t out_pitch) {
  static const int8_t dos[4] = {0, -1, 1, 2};
  for (uint64_t v = 0; v < num_variants; ++v)
    for (uint64_t i = 0; i < num_people; ++i)
      out[v * out_pitch + i] = dos[(rows[v * pitch + i / 4] >> (2 * (i % 4))) & 3];
}

/* ------------------------------------------------------------------------ */
/* Routing restatement (decide.rs)                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  float n_cohort, k_scores, subset_frac, freq;
} route_ctx;

enum { PIVOT = 0, NOPIVOT = 1 };

/* decide.rs:69-100 choose_run_strategy: returns 1 for the frequency-aware tree. */
static int use_complex_tree(const route_ctx* c) {
  if (c->subset_frac <= 0.2750f) return 0;
  if (c->n_cohort <= 2236.0677f) return 0;
  if (c->n_cohort <= 7071.067f) {
    if (c->subset_frac <= 0.7500f) return 0;
    return c->k_scores <= 15.8114f;
  }
  if (c->subset_frac <= 0.7500f) {
    if (c->n_cohort <= 20000.002f) return c->k_scores <= 15.8114f;
    return 1;
  }
  return 1;
}

/* decide.rs:107-216 decide_path_with_freq. */
static int path_with_freq(const route_ctx* c) {
  if (c->n_cohort <= 20000.002f) {
    if (c->freq <= 0.0894f) {
      if (c->freq <= 0.0045f) {
        if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
        return NOPIVOT;
      }
      if (c->n_cohort <= 7071.067f) {
        if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
        return NOPIVOT;
      }
      if (c->subset_frac <= 0.7500f) return NOPIVOT;
      return c->k_scores <= 15.8114f ? PIVOT : NOPIVOT;
    }
    if (c->n_cohort <= 7071.067f) {
      if (c->k_scores <= 15.8114f) {
        if (c->subset_frac <= 0.7500f) {
          if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
          return NOPIVOT;
        }
        return c->n_cohort <= 2236.0677f ? NOPIVOT : PIVOT;
      }
      if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
      return NOPIVOT;
    }
    if (c->subset_frac <= 0.7500f) {
      if (c->k_scores <= 15.8114f) return c->subset_frac <= 0.2750f ? NOPIVOT : PIVOT;
      return NOPIVOT;
    }
    return PIVOT;
  }
  if (c->subset_frac <= 0.2750f) return NOPIVOT;
  if (c->freq <= 0.0045f) return NOPIVOT;
  return PIVOT;
}

/* decide.rs:218-304 decide_path_without_freq. */
static int path_without_freq(const route_ctx* c) {
  if (c->n_cohort <= 20000.002f) {
    if (c->n_cohort <= 7071.067f) {
      if (c->k_scores <= 15.8114f) {
        if (c->subset_frac <= 0.7500f) {
          if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
          return NOPIVOT;
        }
        return NOPIVOT;
      }
      if (c->n_cohort <= 10.0f) return c->subset_frac <= 0.2750f ? PIVOT : NOPIVOT;
      return NOPIVOT;
    }
    if (c->subset_frac <= 0.7500f) return NOPIVOT;
    return PIVOT;
  }
  if (c->subset_frac <= 0.2750f) return NOPIVOT;
  return PIVOT;
}

/* batch.rs:583-614: popcount density with early exit above 0.0894. */
static float density_for_dispatch(const uint8_t* row, uint64_t bpv, uint64_t total_people) {
  if (total_people == 0) return 0.0f;
  uint64_t cutoff = (uint64_t)((float)total_people * 0.0894f);
  uint64_t set = 0, b = 0;
  for (; b + 8 <= bpv; b += 8) {
    uint64_t w;
    memcpy(&w, row + b, 8);
    set += (uint64_t)__builtin_popcountll(w);
    if (set > cutoff) return 1.0f;
  }
  for (; b < bpv; ++b) set += (uint64_t)__builtin_popcount(row[b]);
  return (float)set / (float)total_people;
}

/* ------------------------------------------------------------------------ */
/* Reference CPU engine restatement                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  const uint8_t* rows;
  uint64_t pitch, bpv, total_people, num_people;
  const uint32_t* out_to_fam; /* may be NULL */
  uint64_t K, V;
  const float* w;
  const float* corr;
  const uint32_t* cols;
  const uint64_t* offs;
} ref_job;

static inline uint32_t fam_of(const ref_job* j, uint64_t o) {
  return j->out_to_fam ? j->out_to_fam[o] : (uint32_t)o;
}

/* batch.rs:622-809 + 812-844: variant-major path, f64 direct. */
static void variant_major(const ref_job* j, uint64_t v, double* sums, uint32_t* counts) {
  const uint8_t* row = j->rows + v * j->pitch;
  uint64_t beg = j->offs[v], end = j->offs[v + 1];
  for (uint64_t o = 0; o < j->num_people; ++o) {
    uint32_t f = fam_of(j, o);
    uint32_t g = (row[f >> 2] >> (2 * (f & 3))) & 3u;
    if (g == 0) continue;
    double* s = sums + o * j->K;
    uint32_t* c = counts + o * j->K;
    if (g == 1) {
      for (uint64_t e = beg; e < end; ++e) {
        c[j->cols[e]] += 1;
        s[j->cols[e]] -= (double)j->corr[e];
      }
    } else {
      double dosage = g == 2 ? 1.0 : 2.0;
      for (uint64_t e = beg; e < end; ++e) s[j->cols[e]] += (double)j->w[e] * dosage;
    }
  }
}

/* batch.rs:48-422: person-major path over one dense batch (<= 256 rows).
 * `batch` lists reconciled variant indices; weights/corrections come from a
 * dense [n][K] canvas (pipeline.rs:1648-1662, 1974-1999). */
static void person_major_batch(const ref_job* j, const uint64_t* batch, uint64_t n,
                               float* canvas_w, float* canvas_c, uint8_t* dos,
                               float* acc32, uint16_t* g1, uint16_t* g2, uint16_t* gm,
                               double* sums, uint32_t* counts) {
  uint64_t K = j->K;
  memset(canvas_w, 0, sizeof(float) * n * K);
  memset(canvas_c, 0, sizeof(float) * n * K);
  for (uint64_t r = 0; r < n; ++r) {
    uint64_t v = batch[r];
    for (uint64_t e = j->offs[v]; e < j->offs[v + 1]; ++e) {
      canvas_w[r * K + j->cols[e]] = j->w[e];
      canvas_c[r * K + j->cols[e]] = j->corr[e];
    }
  }
  for (uint64_t o = 0; o < j->num_people; ++o) {
    uint32_t f = fam_of(j, o);
    uint64_t n1 = 0, n2 = 0, nm = 0;
    for (uint64_t r = 0; r < n; ++r) {
      uint32_t g = (j->rows[batch[r] * j->pitch + (f >> 2)] >> (2 * (f & 3))) & 3u;
      dos[r] = (uint8_t)g;
    }
    for (uint64_t r = 0; r < n; ++r) {
      /* pivot_tile: d = hi*(lo+1), missing sentinel for code 01 */
      switch (dos[r]) {
        case 2: g1[n1++] = (uint16_t)r; break;
        case 3: g2[n2++] = (uint16_t)r; break;
        case 1: gm[nm++] = (uint16_t)r; break;
        default: break;
      }
    }
    double* s = sums + o * K;
    uint32_t* c = counts + o * K;
    /* batch.rs:373-385: missing first, CSR order, f64 subtraction */
    for (uint64_t q = 0; q < nm; ++q) {
      uint64_t r = gm[q], v = batch[r];
      for (uint64_t e = j->offs[v]; e < j->offs[v + 1]; ++e) {
        uint32_t col = j->cols[e];
        c[col] += 1;
        s[col] -= (double)canvas_c[r * K + col];
      }
    }
    /* kernel.rs:124-301: f32 lanes; each score is an independent f32 chain */
    for (uint64_t k = 0; k < K; ++k) acc32[k] = 0.0f;
    for (uint64_t q = 0; q < n1; ++q) {
      const float* wr = canvas_w + (uint64_t)g1[q] * K;
      for (uint64_t k = 0; k < K; ++k) acc32[k] = acc32[k] + wr[k];
    }
    for (uint64_t q = 0; q < n2; ++q) {
      const float* wr = canvas_w + (uint64_t)g2[q] * K;
      for (uint64_t k = 0; k < K; ++k) acc32[k] = fmaf(wr[k], 2.0f, acc32[k]);
    }
    for (uint64_t k = 0; k < K; ++k) s[k] += (double)acc32[k];
  }
}

typedef struct {
  const ref_job* job;
  const uint64_t* dense_rows;   /* all dense reconciled indices in order */
  uint64_t n_dense;
  const uint64_t* sparse_rows;
  uint64_t n_sparse;
  int tid, nthreads;
  double* dsum; uint32_t* dcnt;  /* this thread's dense partial   */
  double* ssum; uint32_t* scnt;  /* this thread's sparse partial  */
} worker_arg;

static void* worker(void* p) {
  worker_arg* a = (worker_arg*)p;
  const ref_job* j = a->job;
  uint64_t K = j->K;
  float* cw = (float*)malloc(sizeof(float) * 256 * (K ? K : 1));
  float* cc = (float*)malloc(sizeof(float) * 256 * (K ? K : 1));
  float* acc = (float*)malloc(sizeof(float) * (K ? K : 1));
  uint8_t dos[256];
  uint16_t g1[256], g2[256], gm[256];
  /* dense stream: ChannelBatcher of 256 rows (pipeline.rs:1935); batches are
   * dealt to threads round-robin, each thread folding into its own partial. */
  uint64_t nb = (a->n_dense + 255) / 256;
  for (uint64_t b = (uint64_t)a->tid; b < nb; b += (uint64_t)a->nthreads) {
    uint64_t beg = b * 256, n = a->n_dense - beg < 256 ? a->n_dense - beg : 256;
    person_major_batch(j, a->dense_rows + beg, n, cw, cc, dos, acc, g1, g2, gm, a->dsum, a->dcnt);
  }
  for (uint64_t s = (uint64_t)a->tid; s < a->n_sparse; s += (uint64_t)a->nthreads)
    variant_major(j, a->sparse_rows[s], a->ssum, a->scnt);
  free(cw); free(cc); free(acc);
  return NULL;
}

/* Full restatement of run_single_file_pipeline's arithmetic.
 * rows: reconciled variant v's packed row at rows + v*pitch.
 * baseline: [K] (NULL -> computed from corrections, prepare.rs:644-646).
 * force_path: -1 = route like the reference, 0 = all Pivot, 1 = all NoPivot.
 * Returns 0 on success. */
int oracle_score_reference(const uint8_t* rows, uint64_t pitch, uint64_t bpv,
                           uint64_t total_people, uint64_t num_people,
                           const uint32_t* out_to_fam, uint64_t K, uint64_t V,
                           const float* w, const float* corr, const uint32_t* cols,
                           const uint64_t* offs, const double* baseline,
                           int n_threads, int force_path, double* sums, uint32_t* counts) {
  ref_job j = {rows, pitch, bpv, total_people, num_people, out_to_fam, K, V, w, corr, cols, offs};
  if (n_threads < 1) n_threads = 1;
  uint64_t cells = num_people * K;
  route_ctx rc = {(float)total_people, (float)K,
                  total_people ? (float)num_people / (float)total_people : 0.0f, 0.0f};
  int complex_tree = use_complex_tree(&rc);
  int global_path = path_without_freq(&rc);
  uint64_t* dense = (uint64_t*)malloc(sizeof(uint64_t) * (V ? V : 1));
  uint64_t* sparse = (uint64_t*)malloc(sizeof(uint64_t) * (V ? V : 1));
  uint64_t nd = 0, ns = 0;
  for (uint64_t v = 0; v < V; ++v) {
    int path;
    if (force_path >= 0) {
      path = force_path;
    } else if (complex_tree) {
      route_ctx vc = rc;
      vc.freq = density_for_dispatch(rows + v * pitch, bpv, total_people);
      path = path_with_freq(&vc);
    } else {
      path = global_path;
    }
    if (path == PIVOT) dense[nd++] = v; else sparse[ns++] = v;
  }
  double* part_s = (double*)calloc((size_t)n_threads * 2 * (cells ? cells : 1), sizeof(double));
  uint32_t* part_c = (uint32_t*)calloc((size_t)n_threads * 2 * (cells ? cells : 1), sizeof(uint32_t));
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  worker_arg* args = (worker_arg*)malloc(sizeof(worker_arg) * (size_t)n_threads);
  if (!dense || !sparse || !part_s || !part_c || !th || !args) return -1;
  for (int t = 0; t < n_threads; ++t) {
    worker_arg a = {&j, dense, nd, sparse, ns, t, n_threads,
                    part_s + (size_t)(2 * t) * cells, part_c + (size_t)(2 * t) * cells,
                    part_s + (size_t)(2 * t + 1) * cells, part_c + (size_t)(2 * t + 1) * cells};
    args[t] = a;
    if (n_threads == 1) worker(&args[t]);
    else pthread_create(&th[t], NULL, worker, &args[t]);
  }
  if (n_threads > 1)
    for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
  /* pipeline.rs:1739-1775 baseline broadcast, then counts and sums folded in:
   * sparse partial first, then dense (pipeline.rs:776-791).  Thread partials
   * are reduced in thread order. */
  double* base = (double*)calloc(K ? K : 1, sizeof(double));
  if (baseline) {
    memcpy(base, baseline, sizeof(double) * K);
  } else {
    for (uint64_t e = 0; e < offs[V]; ++e) base[cols[e]] += (double)corr[e];
  }
  for (uint64_t x = 0; x < cells; ++x) {
    double ssum = 0.0, dsum = 0.0;
    uint32_t sc = 0, dc = 0;
    for (int t = 0; t < n_threads; ++t) {
      ssum += part_s[(size_t)(2 * t + 1) * cells + x];
      sc += part_c[(size_t)(2 * t + 1) * cells + x];
      dsum += part_s[(size_t)(2 * t) * cells + x];
      dc += part_c[(size_t)(2 * t) * cells + x];
    }
    double s = base[x % K];
    s += ssum;
    s += dsum;
    sums[x] = s;
    counts[x] = sc + dc;
  }
  free(base); free(dense); free(sparse); free(part_s); free(part_c); free(th); free(args);
  return 0;
}

/* Independent extended-precision scorer: per genotype, x87 long double
 * (64-bit significand), variant order.  sum = baseline + sum_v f(code),
 * f = {00: 0, 01: -corr, 10: w, 11: 2w}; counts = # of 01 over member cells. */
/* Extended-precision scorer: one thread per contiguous range of output
 * people.  Every (person, score) cell is summed over the variants in row
 * order whatever the thread count, so the result does not depend on it. */
typedef struct {
  const uint8_t* rows;
  uint64_t pitch, o0, o1, K, V;
  const uint32_t* out_to_fam;
  const float *w, *corr;
  const uint32_t* cols;
  const uint64_t* offs;
  long double* acc;     /* [o1 - o0][K] */
  uint32_t* counts;     /* caller's [P][K] */
} ExtArgs;

static void* extended_worker(void* p) {
  ExtArgs* a = (ExtArgs*)p;
  const uint64_t K = a->K;
  for (uint64_t v = 0; v < a->V; ++v) {
    const uint8_t* row = a->rows + v * a->pitch;
    const uint64_t e0 = a->offs[v], e1 = a->offs[v + 1];
    if (e0 == e1) continue;
    for (uint64_t o = a->o0; o < a->o1; ++o) {
      uint32_t f = a->out_to_fam ? a->out_to_fam[o] : (uint32_t)o;
      uint32_t g = (row[f >> 2] >> (2 * (f & 3))) & 3u;
      if (g == 0) continue;
      long double* acc = a->acc + (o - a->o0) * K;
      uint32_t* cnt = a->counts + o * K;
      for (uint64_t e = e0; e < e1; ++e) {
        uint32_t k = a->cols[e];
        if (g == 1) { acc[k] -= (long double)a->corr[e]; cnt[k] += 1; }
        else if (g == 2) acc[k] += (long double)a->w[e];
        else acc[k] += 2.0L * (long double)a->w[e];
      }
    }
  }
  return NULL;
}

int oracle_score_extended_mt(const uint8_t* rows, uint64_t pitch, uint64_t num_people,
                             const uint32_t* out_to_fam, uint64_t K, uint64_t V,
                             const float* w, const float* corr, const uint32_t* cols,
                             const uint64_t* offs, const double* baseline,
                             double* sums, uint32_t* counts, int n_threads) {
  uint64_t cells = num_people * K;
  long double* acc = (long double*)calloc(cells ? cells : 1, sizeof(long double));
  if (!acc) return -1;
  for (uint64_t x = 0; x < cells; ++x) counts[x] = 0;
  if (n_threads < 1) n_threads = 1;
  if ((uint64_t)n_threads > num_people) n_threads = num_people ? (int)num_people : 1;
  ExtArgs* args = (ExtArgs*)calloc((size_t)n_threads, sizeof(ExtArgs));
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  if (!args || !th) { free(acc); free(args); free(th); return -1; }
  const uint64_t per = (num_people + (uint64_t)n_threads - 1) / (uint64_t)n_threads;
  for (int t = 0; t < n_threads; ++t) {
    ExtArgs* a = &args[t];
    a->rows = rows; a->pitch = pitch; a->K = K; a->V = V; a->out_to_fam = out_to_fam;
    a->w = w; a->corr = corr; a->cols = cols; a->offs = offs; a->counts = counts;
    a->o0 = (uint64_t)t * per < num_people ? (uint64_t)t * per : num_people;
    a->o1 = a->o0 + per < num_people ? a->o0 + per : num_people;
    a->acc = acc + a->o0 * K;
  }
  int spawned = 0;
  for (int t = 1; t < n_threads; ++t) {
    if (pthread_create(&th[t], NULL, extended_worker, &args[t]) != 0) break;
    spawned = t;
  }
  extended_worker(&args[0]);
  for (int t = 1; t <= spawned; ++t) pthread_join(th[t], NULL);
  for (int t = spawned + 1; t < n_threads; ++t) extended_worker(&args[t]);
  for (uint64_t x = 0; x < cells; ++x) {
    long double b = 0.0L;
    if (baseline) b = (long double)baseline[x % K];
    sums[x] = (double)(b + acc[x]);
  }
  if (!baseline) {
    long double* base = (long double*)calloc(K ? K : 1, sizeof(long double));
    for (uint64_t e = 0; e < offs[V]; ++e) base[cols[e]] += (long double)corr[e];
    for (uint64_t x = 0; x < cells; ++x) sums[x] = (double)(base[x % K] + acc[x]);
    free(base);
  }
  free(args);
  free(th);
  free(acc);
  return 0;
}

int oracle_score_extended(const uint8_t* rows, uint64_t pitch, uint64_t num_people,
                          const uint32_t* out_to_fam, uint64_t K, uint64_t V,
                          const float* w, const float* corr, const uint32_t* cols,
                          const uint64_t* offs, const double* baseline,
                          double* sums, uint32_t* counts) {
  return oracle_score_extended_mt(rows, pitch, num_people, out_to_fam, K, V, w, corr, cols, offs,
                                  baseline, sums, counts, 1);
}

/* Extended-precision gradient for the backward check (dense over all cells):
 * gw[v*K+k] = sum_p d'(p,v) * gs[p*K+k], d' = dosage with missing -> 0,
 * gc[v*K+k] = -sum_{p missing} gs[p*K+k]. */
int oracle_backward_extended(const uint8_t* rows, uint64_t pitch, uint64_t num_people,
                             const uint32_t* out_to_fam, uint64_t K, uint64_t V,
                             const uint32_t* cols, const uint64_t* offs,
                             const float* gs, double* gw, double* gc) {
  long double* tw = (long double*)malloc(sizeof(long double) * (K ? K : 1));
  long double* tc = (long double*)malloc(sizeof(long double) * (K ? K : 1));
  if (!tw || !tc) return -1;
  for (uint64_t v = 0; v < V; ++v) {
    const uint8_t* row = rows + v * pitch;
    for (uint64_t k = 0; k < K; ++k) { tw[k] = 0.0L; tc[k] = 0.0L; }
    for (uint64_t o = 0; o < num_people; ++o) {
      uint32_t f = out_to_fam ? out_to_fam[o] : (uint32_t)o;
      uint32_t g = (row[f >> 2] >> (2 * (f & 3))) & 3u;
      if (g == 0) continue;
      const float* gp = gs + o * K;
      if (g == 1) { for (uint64_t k = 0; k < K; ++k) tc[k] -= (long double)gp[k]; }
      else if (g == 2) { for (uint64_t k = 0; k < K; ++k) tw[k] += (long double)gp[k]; }
      else { for (uint64_t k = 0; k < K; ++k) tw[k] += 2.0L * (long double)gp[k]; }
    }
    for (uint64_t k = 0; k < K; ++k) {
      gw[v * K + k] = (double)tw[k];
      if (gc) gc[v * K + k] = (double)tc[k];
    }
  }
  free(tw); free(tc);
  return 0;
}
