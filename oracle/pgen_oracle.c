/* pgen_oracle.c — TEST INFRASTRUCTURE ONLY: a C restatement of the .pgen
 * hard-call decode into .bed rows, for timing a compiled CPU decoder beside
 * the GPU one (bench.py's CPU-baseline leg) and as a second checker.
 *
 * It follows oracle/pgen_oracle.py step for step (that file cites the
 * reference, shared/adapt_plink2.rs, per function):
 *   header and index (:1512-1716), varints (:1721-1741), difflists
 *   (:1920-2040), LD anchors per 2^16-variant block (:2237-2257), main-track
 *   types 0-4, 6, 7 and the type-3 swap (:2574-2666), categories -> .bed
 *   codes of the A1 = ALT dosage with padding fields 01 (:927-935,
 *   :1136-1158).
 * Records with multiallelic or dosage tracks, type 5, LD records without an
 * anchor, and malformed difflists (overruns, group-length mismatches, ids
 * that do not rise) are errors.
 *
 * Work: non-LD records in parallel over `threads` host threads, then the LD
 * records from their anchors' rows (read back as categories). */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t m, n;
  uint64_t* offs;
  uint32_t* lens;
  uint8_t* types;
  uint32_t* anchor;   /* LD record's anchor, else UINT32_MAX */
} pg_index;

static const uint8_t kCatToBed[4] = {3, 2, 0, 1};
static const uint8_t kBedToCat[4] = {2, 3, 1, 0};

static uint64_t le(const uint8_t* p, int bytes) {
  uint64_t v = 0;
  for (int i = 0; i < bytes; ++i) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

static void free_index(pg_index* ix) {
  free(ix->offs);
  free(ix->lens);
  free(ix->types);
  free(ix->anchor);
}

static int parse(const uint8_t* d, uint64_t len, pg_index* ix) {
  memset(ix, 0, sizeof *ix);
  if (len < 12 || d[0] != 0x6C || d[1] != 0x1B) return -1;
  const uint8_t mode = d[2];
  const uint64_t m = le(d + 3, 4), n = le(d + 7, 4);
  ix->m = m;
  ix->n = n;
  ix->offs = calloc(m ? m : 1, 8);
  ix->lens = calloc(m ? m : 1, 4);
  ix->types = calloc(m ? m : 1, 1);
  ix->anchor = calloc(m ? m : 1, 4);
  if (!ix->offs || !ix->lens || !ix->types || !ix->anchor) return -2;
  if (mode == 0x02) {
    /* body after 13 bytes (+ reference flags), adapt_plink2.rs:2048-2057 */
    const uint64_t rec = (n + 3) / 4;
    const uint64_t base = 13 + (((d[11] >> 6) & 3) == 3 ? (m + 7) / 8 : 0);
    for (uint64_t v = 0; v < m; ++v) {
      ix->offs[v] = base + v * rec;
      ix->lens[v] = (uint32_t)rec;
    }
  } else if (mode == 0x10 || mode == 0x11) {
    const uint8_t fmt = d[11];
    const int type_bits = (fmt & 0x0F) <= 3 ? 4 : 8;
    const int len_bytes = (fmt & 0x07) % 4 + 1;
    const int ac_tab[4] = {0, 1, 2, 4};
    const int ac_bytes = ac_tab[(fmt >> 4) & 3];
    const int ref_flag_mode = (fmt >> 6) & 3;
    const uint64_t blocks = (m + 0xFFFF) >> 16;
    uint64_t off = 12;
    if (off + 8 * blocks > len) return -1;
    uint64_t idx = 0;
    for (uint64_t b = 0; b < blocks; ++b) {
      const uint64_t cnt = m - idx < 65536 ? m - idx : 65536;
      const uint64_t tbytes = type_bits == 4 ? (cnt + 1) / 2 : cnt;
      const uint64_t need = tbytes + cnt * len_bytes + cnt * ac_bytes +
                            (ref_flag_mode == 3 ? (cnt + 7) / 8 : 0);
      uint64_t at = off + 8 * blocks;
      for (uint64_t bb = 0; bb < b; ++bb) {   /* skip earlier blocks' arrays */
        const uint64_t c = m - (bb << 16) < 65536 ? m - (bb << 16) : 65536;
        at += (type_bits == 4 ? (c + 1) / 2 : c) + c * len_bytes + c * ac_bytes +
              (ref_flag_mode == 3 ? (c + 7) / 8 : 0);
      }
      if (at + need > len) return -1;
      for (uint64_t i = 0; i < cnt; ++i)
        ix->types[idx + i] = type_bits == 4 ? (uint8_t)((d[at + i / 2] >> (4 * (i % 2))) & 0x0F)
                                            : d[at + i];
      at += tbytes;
      uint64_t rec_off = le(d + off + 8 * b, 8);
      for (uint64_t i = 0; i < cnt; ++i) {
        ix->lens[idx + i] = (uint32_t)le(d + at + i * len_bytes, len_bytes);
        ix->offs[idx + i] = rec_off;
        rec_off += ix->lens[idx + i];
      }
      idx += cnt;
    }
  } else {
    return -1;
  }
  int64_t last = -1;
  for (uint64_t v = 0; v < m; ++v) {
    if (ix->offs[v] > len || ix->offs[v] + ix->lens[v] > len) return -1;
    if (ix->types[v] & 0xE8u) return -1;
    const uint32_t kind = ix->types[v] & 7u;
    if (kind == 5) return -1;
    if ((v & 0xFFFF) == 0) last = -1;
    if (kind == 2 || kind == 3) {
      if (last < 0) return -1;
      ix->anchor[v] = (uint32_t)last;
    } else {
      ix->anchor[v] = UINT32_MAX;
      last = (int64_t)v;
    }
  }
  return 0;
}

static int varint(const uint8_t* p, uint32_t len, uint32_t* cur, uint64_t* out) {
  uint64_t v = 0;
  for (uint32_t shift = 0; shift < 64; shift += 7) {
    if (*cur >= len) return -1;
    const uint8_t b = p[(*cur)++];
    v |= (uint64_t)(b & 0x7F) << shift;
    if (!(b & 0x80)) {
      *out = v;
      return 0;
    }
  }
  return -1;
}

/* Apply the difflist at `cur` to cats[n]. */
static int difflist(const uint8_t* p, uint32_t len, uint32_t cur, uint64_t n, uint8_t* cats) {
  uint64_t l;
  if (varint(p, len, &cur, &l)) return -1;
  if (l == 0) return 0;
  const uint64_t groups = (l + 63) / 64;
  const int wid = n <= (1u << 8) ? 1 : n <= (1u << 16) ? 2 : n <= (1u << 24) ? 3 : 4;
  const uint64_t first_at = cur, glen_at = first_at + groups * wid, vals_at = glen_at + groups - 1;
  uint64_t at = vals_at + (l + 3) / 4;
  if (at > len) return -1;
  for (uint64_t g = 0; g < groups; ++g) {
    const uint64_t count = g + 1 < groups ? 64 : l - 64 * (groups - 1);
    uint64_t id = le(p + first_at + g * wid, wid);
    const uint64_t start = at;
    for (uint64_t e = 0; e < count; ++e) {
      if (e > 0) {
        uint64_t dl;
        uint32_t c32 = (uint32_t)at;
        if (varint(p, len, &c32, &dl) || dl == 0) return -1;
        at = c32;
        id += dl;
      }
      const uint64_t idx = 64 * g + e;
      const uint8_t val = (p[vals_at + idx / 4] >> (2 * (idx % 4))) & 3;
      if (id < n) cats[id] = val;
    }
    if (g + 1 < groups) {
      if (at - start != (uint64_t)p[glen_at + g] + 63) return -1;
      if (id >= le(p + first_at + (g + 1) * wid, wid)) return -1;
    }
  }
  return 0;
}

static void pack(const uint8_t* cats, uint64_t n, uint8_t* row) {
  const uint64_t bpv = (n + 3) / 4;
  for (uint64_t j = 0; j < bpv; ++j) {
    uint8_t b = 0;
    for (int k = 0; k < 4; ++k) {
      const uint64_t i = 4 * j + k;
      b |= (uint8_t)((i < n ? kCatToBed[cats[i]] : 1) << (2 * k));
    }
    row[j] = b;
  }
}

static int decode_one(const uint8_t* d, const pg_index* ix, uint64_t v, uint8_t* rows,
                      uint64_t pitch, uint8_t* cats) {
  const uint8_t* p = d + ix->offs[v];
  const uint32_t len = ix->lens[v];
  const uint32_t kind = ix->types[v] & 7u;
  const uint64_t n = ix->n, bpv = (n + 3) / 4;
  uint32_t cur = 0;
  if (kind == 0) {
    if (len < bpv) return -1;
    for (uint64_t i = 0; i < n; ++i) cats[i] = (p[i / 4] >> (2 * (i % 4))) & 3;
    pack(cats, n, rows + v * pitch);
    return 0;
  }
  if (kind == 1) {
    static const int8_t lo[16] = {-1, 0, 0, 0, -1, 1, 1, -1, -1, 2, -1, -1, -1, -1, -1, -1};
    static const int8_t hi[16] = {-1, 1, 2, 3, -1, 2, 3, -1, -1, 3, -1, -1, -1, -1, -1, -1};
    if (len < 1 || p[0] >= 16 || lo[p[0]] < 0) return -1;
    const uint64_t nb = (n + 7) / 8;
    if (len < 1 + nb) return -1;
    for (uint64_t i = 0; i < n; ++i)
      cats[i] = (uint8_t)(((p[1 + i / 8] >> (i % 8)) & 1) ? hi[p[0]] : lo[p[0]]);
    cur = (uint32_t)(1 + nb);
  } else if (kind == 2 || kind == 3) {
    const uint8_t* a = rows + (uint64_t)ix->anchor[v] * pitch;
    for (uint64_t i = 0; i < n; ++i) cats[i] = kBedToCat[(a[i / 4] >> (2 * (i % 4))) & 3];
  } else if (kind == 4 || kind == 6 || kind == 7) {
    memset(cats, kind == 4 ? 0 : kind == 6 ? 2 : 3, n);
  } else {
    return -1;
  }
  if (difflist(p, len, cur, n, cats)) return -1;
  if (kind == 3)
    for (uint64_t i = 0; i < n; ++i)
      if (!(cats[i] & 1)) cats[i] ^= 2;
  pack(cats, n, rows + v * pitch);
  return 0;
}

typedef struct {
  const uint8_t* d;
  const pg_index* ix;
  uint8_t* rows;
  uint64_t pitch, v0, v1;
  int ld;    /* pass: 0 = non-LD records, 1 = LD records */
  int err;
} pg_job;

static void* run_job(void* arg) {
  pg_job* j = arg;
  uint8_t* cats = malloc(j->ix->n ? j->ix->n : 1);
  if (!cats) {
    j->err = -2;
    return NULL;
  }
  for (uint64_t v = j->v0; v < j->v1 && !j->err; ++v) {
    const int is_ld = j->ix->anchor[v] != UINT32_MAX;
    if (is_ld == j->ld && decode_one(j->d, j->ix, v, j->rows, j->pitch, cats)) j->err = -1;
  }
  free(cats);
  return NULL;
}

/* Header counts; 0 or -1 (not a supported .pgen). */
int pgen_oracle_dims(const uint8_t* data, uint64_t len, uint64_t* variants, uint64_t* samples) {
  pg_index ix;
  const int rc = parse(data, len, &ix);
  if (!rc) {
    *variants = ix.m;
    *samples = ix.n;
  }
  free_index(&ix);
  return rc;
}

/* Decode every variant into rows[v * pitch ..] (ceil(samples/4) bytes each).
 * 0 on success, -1 for a malformed or unsupported file. */
int pgen_oracle_decode(const uint8_t* data, uint64_t len, uint8_t* rows, uint64_t pitch,
                       int threads) {
  pg_index ix;
  int rc = parse(data, len, &ix);
  if (rc) {
    free_index(&ix);
    return rc;
  }
  if (threads < 1) threads = 1;
  if ((uint64_t)threads > ix.m) threads = ix.m ? (int)ix.m : 1;
  pg_job* jobs = calloc((size_t)threads, sizeof *jobs);
  pthread_t* tid = calloc((size_t)threads, sizeof *tid);
  if (!jobs || !tid) {
    free(jobs);
    free(tid);
    free_index(&ix);
    return -2;
  }
  for (int pass = 0; pass < 2 && !rc; ++pass) {
    const uint64_t per = (ix.m + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
      const uint64_t v0 = per * t, v1 = per * (t + 1) < ix.m ? per * (t + 1) : ix.m;
      jobs[t] = (pg_job){data, &ix, rows, pitch, v0 < ix.m ? v0 : ix.m, v1, pass, 0};
      pthread_create(&tid[t], NULL, run_job, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) {
      pthread_join(tid[t], NULL);
      if (jobs[t].err) rc = jobs[t].err;
    }
  }
  free(jobs);
  free(tid);
  free_index(&ix);
  return rc;
}
