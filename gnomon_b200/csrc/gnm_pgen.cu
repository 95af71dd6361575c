// gnm_pgen.cu — PLINK 2 .pgen hard calls -> PLINK 1 .bed rows on the device.
//
// gnomon reads a .pgen through a "virtual .bed" (shared/adapt_plink2.rs): every
// variant's hard calls are decoded into genotype categories (0 hom REF, 1 het,
// 2 hom ALT, 3 missing) and packed as the .bed codes of the A1 = ALT dosage
// (shared/adapt_plink2.rs:927-935, 1136-1158): 2 -> 00, 1 -> 10, 0 -> 11,
// missing -> 01, padding fields past the last sample -> 01.  The scoring
// engines then read those rows unchanged.  This file does the same decode on
// the GPU, straight into the engines' row layout.
//
// Supported: storage modes 0x02 (fixed-width hard calls) and 0x10 / 0x11
// (variable-width) with biallelic records whose main track is type 0 (2-bit),
// 1 (two categories as a bit array + difflist), 2 / 3 (LD-compressed against
// the most recent non-LD record of the same 2^16-variant block; 3 swaps REF and
// ALT homozygotes after the patch) or 4 / 6 / 7 (all hom REF / hom ALT /
// missing + difflist) — shared/adapt_plink2.rs:2237-2257, 2574-2666.  Phase
// tracks follow the main track and do not change hard calls.  Records with
// multiallelic or dosage tracks are rejected (the reference projects or
// coerces them; this decoder does not).
//
// Layout of the work: the bijection category -> .bed code lets every step
// run on .bed codes directly.  Kernel 1 decodes the non-LD records (one CTA
// per variant: a LUT pass over the 2-bit or 1-bit array, or a fill), kernel 2
// the LD-compressed ones from their anchors' rows.  A record's difflist is
// parsed once (thread 0: length, first sample ids, group byte lengths), then
// its groups of 64 entries are applied in parallel, one thread per group,
// each walking its base-128 sample-id deltas and patching 2-bit fields with
// 32-bit atomics (fields of one word may belong to different groups).
// Every byte read is bounded by the record's length; a malformed record sets
// the error word and its row is left incomplete.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gnm_plan.h"

namespace gnm {
namespace {

constexpr uint32_t kPgThreads = 256;
constexpr uint32_t kPgChunk = 2048;               // difflist groups laid out per round
constexpr uint64_t kPgMaxSamples = uint64_t(1) << 31;

enum : uint32_t { kPgErrBounds = 1u, kPgErrPair = 2u };

constexpr uint32_t kNoAnchor = 0xFFFFFFFFu;

struct PgArgs {
  const uint8_t* pgen;         // whole file
  const uint64_t* offsets;     // [V] record offsets
  const uint32_t* lens;        // [V] record lengths
  const uint8_t* types;        // [V] record types
  const uint32_t* anchor_of;   // [V] anchor of an LD-compressed record, else kNoAnchor
  uint32_t begin, count;       // variants [begin, begin + count) -> rows 0 .. count - 1
  uint32_t extra;              // a non-LD variant before `begin` decoded into `scratch`
  uint64_t n;                  // samples
  uint8_t* rows;               // [count][pitch] .bed rows
  uint64_t pitch;
  uint8_t* scratch;            // one row: the anchor of the range's first LD records
  uint32_t* err;               // [0] error bits, [1] first bad variant (atomicMin)
};

__constant__ uint8_t kCatToBed[4] = {0x3, 0x2, 0x0, 0x1};

__device__ __forceinline__ void flag(const PgArgs& a, uint32_t bit, uint32_t v) {
  atomicOr(a.err, bit);
  atomicMin(a.err + 1, v);
}

// Bounded record reader: every read checks the record length.
struct Rec {
  const uint8_t* p;
  uint32_t len;
  __device__ bool byte(uint32_t at, uint32_t& out) const {
    if (at >= len) return false;
    out = p[at];
    return true;
  }
  __device__ bool varint(uint32_t& cur, uint64_t& out) const {
    out = 0;
    for (uint32_t shift = 0; shift < 64; shift += 7) {
      uint32_t b;
      if (!byte(cur++, b)) return false;
      out |= uint64_t(b & 0x7Fu) << shift;
      if (!(b & 0x80u)) return true;
    }
    return false;
  }
};

// Set the 2-bit .bed code of sample `id` in a row (other fields untouched).
__device__ __forceinline__ void put_code(uint8_t* row, uint64_t id, uint32_t code) {
  uint32_t* w = reinterpret_cast<uint32_t*>(row) + id / 16;
  const uint32_t sh = 2 * uint32_t(id % 16);
  atomicAnd(w, ~(3u << sh));
  atomicOr(w, code << sh);
}

// Apply the difflist that starts at `cur` (all threads of the CTA call this).
// Layout (shared/adapt_plink2.rs:1920-2040): length (varint); one first sample
// id per group of 64 entries (1-4 bytes by sample count); the byte lengths of
// all but the last group's deltas, minus 63; the 2-bit values; the groups'
// base-128 id deltas.  Thread 0 lays out up to kPgChunk groups at a time, the
// CTA applies them, one thread per group.
__device__ void apply_difflist(const PgArgs& a, const Rec& r, uint32_t cur, uint8_t* row,
                               uint32_t v) {
  __shared__ uint32_t s_len, s_groups, s_wid, s_first_at, s_glen_at, s_vals, s_next, s_ok;
  __shared__ uint32_t s_start[kPgChunk];   // byte offset of a group's deltas
  __shared__ uint32_t s_first[kPgChunk];   // a group's first sample id
  if (threadIdx.x == 0) {
    s_ok = 1u;
    uint64_t l = 0;
    if (!r.varint(cur, l) || l > a.n) {
      s_ok = 0u;
      flag(a, kPgErrBounds, v);
    } else {
      const uint32_t groups = uint32_t((l + 63) / 64);
      const uint32_t wid = a.n <= (1u << 8) ? 1 : a.n <= (1u << 16) ? 2 : a.n <= (1u << 24) ? 3 : 4;
      s_len = uint32_t(l);
      s_groups = groups;
      s_wid = wid;
      s_first_at = cur;
      s_glen_at = cur + groups * wid;
      s_vals = s_glen_at + (groups > 0 ? groups - 1 : 0);
      s_next = s_vals + uint32_t((l + 3) / 4);
      if (s_next > r.len) {
        s_ok = 0u;
        flag(a, kPgErrBounds, v);
      }
    }
  }
  __syncthreads();
  if (!s_ok) return;
  const uint32_t len = s_len, groups = s_groups;
  for (uint32_t c0 = 0; c0 < groups; c0 += kPgChunk) {
    const uint32_t cn = min(kPgChunk, groups - c0);
    if (threadIdx.x == 0) {
      uint32_t at = s_next;
      for (uint32_t i = 0; i < cn && s_ok; ++i) {
        const uint32_t g = c0 + i;
        uint32_t id = 0;
        for (uint32_t k = 0; k < s_wid; ++k) {
          uint32_t b;
          if (!r.byte(s_first_at + g * s_wid + k, b)) {
            s_ok = 0u;
            break;
          }
          id |= b << (8 * k);
        }
        s_first[i] = id;
        s_start[i] = at;
        if (g + 1 < groups) {
          uint32_t b = 0;
          if (!r.byte(s_glen_at + g, b)) s_ok = 0u;
          at += b + 63;
        }
      }
      s_next = at;
      if (!s_ok) flag(a, kPgErrBounds, v);
    }
    __syncthreads();
    if (!s_ok) return;
    for (uint32_t i = threadIdx.x; i < cn; i += blockDim.x) {
      const uint32_t g = c0 + i;
      const uint32_t count = g + 1 < groups ? 64u : len - 64u * (groups - 1);
      uint64_t id = s_first[i];
      uint32_t at = s_start[i];
      for (uint32_t e = 0; e < count; ++e) {
        if (e > 0) {
          uint64_t d;
          if (!r.varint(at, d)) {
            flag(a, kPgErrBounds, v);
            break;
          }
          id += d;
        }
        const uint32_t idx = 64 * g + e;
        const uint32_t val = (r.p[s_vals + idx / 4] >> (2 * (idx % 4))) & 3u;
        if (id < a.n) put_code(row, id, kCatToBed[val]);
      }
    }
    __syncthreads();   // before thread 0 lays out the next chunk
  }
}

// Padding fields of the last byte -> 01 (missing), as the reference packs them.
__device__ __forceinline__ void fix_tail(const PgArgs& a, uint8_t* row) {
  const uint32_t rem = uint32_t(a.n % 4);
  if (threadIdx.x == 0 && rem) {
    const uint64_t last = (a.n + 3) / 4 - 1;
    uint32_t b = row[last];
    for (uint32_t k = rem; k < 4; ++k) b = (b & ~(3u << (2 * k))) | (1u << (2 * k));
    row[last] = uint8_t(b);
  }
}

// One CTA per variant of the range (LD-compressed ones return at once), plus
// one CTA for `extra` when the range's first LD records anchor before it.
__global__ void __launch_bounds__(kPgThreads) gnm_pgen_direct(PgArgs a) {
  __shared__ uint8_t lut[256];
  const bool in_range = blockIdx.x < a.count;
  const uint32_t v = in_range ? a.begin + blockIdx.x : a.extra;
  if (a.anchor_of[v] != kNoAnchor) return;
  const Rec r{a.pgen + a.offsets[v], a.lens[v]};
  const uint32_t kind = a.types[v] & 7u;
  uint8_t* row = in_range ? a.rows + uint64_t(blockIdx.x) * a.pitch : a.scratch;
  const uint64_t bpv = (a.n + 3) / 4;
  uint32_t cur = 0;
  if (kind == 0) {
    // byte of four PGEN 2-bit categories -> byte of four .bed codes
    for (uint32_t x = threadIdx.x; x < 256; x += blockDim.x) {
      uint32_t o = 0;
      for (uint32_t k = 0; k < 4; ++k) o |= uint32_t(kCatToBed[(x >> (2 * k)) & 3u]) << (2 * k);
      lut[x] = uint8_t(o);
    }
    __syncthreads();
    if (r.len < bpv) {
      if (threadIdx.x == 0) flag(a, kPgErrBounds, v);
      return;
    }
    for (uint64_t j = threadIdx.x; j < bpv; j += blockDim.x) row[j] = lut[r.p[j]];
    __syncthreads();
    fix_tail(a, row);
    return;
  }
  if (kind == 1) {
    // pair code -> (low, high) categories; bit set = high
    uint32_t pc = 0;
    const bool okb = r.byte(0, pc);
    int low = -1, high = -1;
    switch (pc) {
      case 1: low = 0; high = 1; break;
      case 2: low = 0; high = 2; break;
      case 3: low = 0; high = 3; break;
      case 5: low = 1; high = 2; break;
      case 6: low = 1; high = 3; break;
      case 9: low = 2; high = 3; break;
      default: break;
    }
    if (!okb || low < 0) {
      if (threadIdx.x == 0) flag(a, kPgErrPair, v);
      return;
    }
    const uint32_t nb = uint32_t((a.n + 7) / 8);
    if (r.len < 1 + nb) {
      if (threadIdx.x == 0) flag(a, kPgErrBounds, v);
      return;
    }
    // nibble of four bits -> byte of four .bed codes
    for (uint32_t x = threadIdx.x; x < 16; x += blockDim.x) {
      uint32_t o = 0;
      for (uint32_t k = 0; k < 4; ++k)
        o |= uint32_t(kCatToBed[((x >> k) & 1u) ? high : low]) << (2 * k);
      lut[x] = uint8_t(o);
    }
    __syncthreads();
    for (uint64_t j = threadIdx.x; j < bpv; j += blockDim.x)
      row[j] = lut[(r.p[1 + j / 2] >> (4 * (j % 2))) & 15u];
    cur = 1 + nb;
  } else if (kind == 4 || kind == 6 || kind == 7) {
    const uint32_t c = kCatToBed[kind == 4 ? 0 : kind == 6 ? 2 : 3];
    for (uint64_t j = threadIdx.x; j < bpv; j += blockDim.x) row[j] = uint8_t(c * 0x55u);
  } else {
    if (threadIdx.x == 0) flag(a, kPgErrPair, v);
    return;
  }
  __syncthreads();
  apply_difflist(a, r, cur, row, v);
  __syncthreads();
  fix_tail(a, row);
}

// One CTA per variant of the range (non-LD ones return at once).  The anchor
// row is in the range's rows, or in `scratch` when it precedes the range.
__global__ void __launch_bounds__(kPgThreads) gnm_pgen_ld(PgArgs a) {
  const uint32_t v = a.begin + blockIdx.x;
  const uint32_t anchor = a.anchor_of[v];
  if (anchor == kNoAnchor) return;
  const Rec r{a.pgen + a.offsets[v], a.lens[v]};
  const uint32_t kind = a.types[v] & 7u;
  uint8_t* row = a.rows + uint64_t(blockIdx.x) * a.pitch;
  const uint8_t* src =
      anchor >= a.begin ? a.rows + uint64_t(anchor - a.begin) * a.pitch : a.scratch;
  const uint64_t bpv = (a.n + 3) / 4;
  const uint64_t words = bpv / 4;   // whole 32-bit words; the rest byte by byte
  const uint32_t* s32 = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d32 = reinterpret_cast<uint32_t*>(row);
  for (uint64_t j = threadIdx.x; j < words; j += blockDim.x) d32[j] = s32[j];
  for (uint64_t j = 4 * words + threadIdx.x; j < bpv; j += blockDim.x) row[j] = src[j];
  __syncthreads();
  apply_difflist(a, r, 0, row, v);
  __syncthreads();
  if (kind == 3) {
    // swap hom REF (11) and hom ALT (00): flip both bits of fields whose bits agree
    for (uint64_t j = threadIdx.x; j < words; j += blockDim.x) {
      const uint32_t x = d32[j];
      const uint32_t same = ~(x ^ (x >> 1)) & 0x55555555u;
      d32[j] = x ^ (same | (same << 1));
    }
    for (uint64_t j = 4 * words + threadIdx.x; j < bpv; j += blockDim.x) {
      const uint32_t x = row[j];
      const uint32_t same = ~(x ^ (x >> 1)) & 0x55u;
      row[j] = uint8_t(x ^ (same | (same << 1)));
    }
    __syncthreads();
  }
  fix_tail(a, row);
}

// ---- host ----------------------------------------------------------------------

struct PgenIndex {
  uint64_t variants = 0, samples = 0;
  std::vector<uint64_t> offsets;
  std::vector<uint32_t> lens;
  std::vector<uint8_t> types;
};

uint64_t le(const uint8_t* p, int bytes) {
  uint64_t v = 0;
  for (int i = 0; i < bytes; ++i) v |= uint64_t(p[i]) << (8 * i);
  return v;
}

// Header of a .pgen (shared/adapt_plink2.rs:1512-1716): per-variant record
// offsets, lengths and types.  Validates everything the kernels rely on.
PgenIndex parse_pgen(const uint8_t* d, uint64_t len) {
  if (!d || len < 12 || d[0] != 0x6C || d[1] != 0x1B) fail(GNM_ERR_IO, "not a .pgen (bad magic)");
  PgenIndex ix;
  const uint8_t mode = d[2];
  ix.variants = le(d + 3, 4);
  ix.samples = le(d + 7, 4);
  if (ix.samples == 0 || ix.samples > kPgMaxSamples)
    fail(GNM_ERR_INVALID, ".pgen sample count must be 1.." + std::to_string(kPgMaxSamples));
  const uint64_t m = ix.variants;
  ix.offsets.resize(m);
  ix.lens.resize(m);
  ix.types.assign(m, 0);
  if (mode == 0x02) {
    const uint64_t rec = (ix.samples + 3) / 4;
    for (uint64_t v = 0; v < m; ++v) {
      ix.offsets[v] = 12 + v * rec;
      ix.lens[v] = uint32_t(rec);
    }
  } else if (mode == 0x10 || mode == 0x11) {
    const uint8_t fmt = d[11];
    const int type_bits = (fmt & 0x0F) <= 3 ? 4 : 8;
    const int len_bytes = (fmt & 0x07) % 4 + 1;
    const int ac_bytes = (int[]){0, 1, 2, 4}[(fmt >> 4) & 3];
    const int ref_flag_mode = (fmt >> 6) & 3;
    const uint64_t blocks = (m + 0xFFFF) >> 16;
    uint64_t off = 12;
    if (off + 8 * blocks > len) fail(GNM_ERR_IO, "truncated .pgen header");
    std::vector<uint64_t> block_off(blocks);
    for (uint64_t b = 0; b < blocks; ++b, off += 8) block_off[b] = le(d + off, 8);
    for (uint64_t b = 0, idx = 0; b < blocks; ++b) {
      const uint64_t cnt = std::min<uint64_t>(m - idx, 1 << 16);
      const uint64_t tbytes = type_bits == 4 ? (cnt + 1) / 2 : cnt;
      const uint64_t need = tbytes + cnt * len_bytes + cnt * ac_bytes +
                            (ref_flag_mode == 3 ? (cnt + 7) / 8 : 0);
      if (off + need > len) fail(GNM_ERR_IO, "truncated .pgen header");
      for (uint64_t i = 0; i < cnt; ++i)
        ix.types[idx + i] =
            type_bits == 4 ? uint8_t((d[off + i / 2] >> (4 * (i % 2))) & 0x0F) : d[off + i];
      off += tbytes;
      uint64_t rec_off = block_off[b];
      for (uint64_t i = 0; i < cnt; ++i) {
        ix.lens[idx + i] = uint32_t(le(d + off + i * len_bytes, len_bytes));
        ix.offsets[idx + i] = rec_off;
        rec_off += ix.lens[idx + i];
      }
      off += cnt * len_bytes + cnt * ac_bytes + (ref_flag_mode == 3 ? (cnt + 7) / 8 : 0);
      idx += cnt;
    }
  } else {
    char buf[64];
    std::snprintf(buf, sizeof buf, "unsupported .pgen storage mode 0x%02x", mode);
    fail(GNM_ERR_INVALID, buf);
  }
  for (uint64_t v = 0; v < m; ++v) {
    if (ix.offsets[v] + ix.lens[v] > len || ix.offsets[v] > len)
      fail(GNM_ERR_IO, "truncated .pgen: record " + std::to_string(v) + " lies past the end");
    if (ix.types[v] & 0xE8u)
      fail(GNM_ERR_INVALID, "variant " + std::to_string(v) +
                                ": multiallelic or dosage tracks are not supported");
    const uint32_t kind = ix.types[v] & 7u;
    if (kind == 5) fail(GNM_ERR_INVALID, "variant " + std::to_string(v) + ": main-track type 5");
  }
  return ix;
}

}  // namespace

}  // namespace gnm

// A .pgen resident on one device: the file's bytes, its record index and the
// LD anchor of every record, plus a sticky error word the kernels set.
struct gnm_pgen {
  int device = 0;
  uint64_t variants = 0, samples = 0, file_bytes = 0, device_bytes = 0;
  std::vector<uint32_t> anchor_of;   // host copy: the range's out-of-range anchor
  std::vector<void*> bufs;
  gnm::PgArgs base{};
  ~gnm_pgen() {
    for (void* x : bufs) gnm::pool_free(x);
  }
};

namespace gnm {

static gnm_pgen* pgen_open_impl(const uint8_t* pgen, uint64_t pgen_len, int device) {
  PgenIndex ix = parse_pgen(pgen, pgen_len);
  const uint64_t m = ix.variants;
  // one CTA per variant: the grid's x extent bounds the variant count
  if (m > 0x7FFFFFFEull) fail(GNM_ERR_INVALID, "more than 2^31 - 2 .pgen variants");
  // LD-compressed records diff against the most recent non-LD record of their
  // 2^16-variant block (shared/adapt_plink2.rs:2237-2257)
  std::vector<uint32_t> anchor_of(m, kNoAnchor);
  int64_t last = -1;
  for (uint64_t v = 0; v < m; ++v) {
    if ((v & 0xFFFF) == 0) last = -1;
    const uint32_t kind = ix.types[v] & 7u;
    if (kind == 2 || kind == 3) {
      if (last < 0)
        fail(GNM_ERR_IO, "variant " + std::to_string(v) + ": LD-compressed record without an "
                                                           "anchor in its block");
      anchor_of[v] = uint32_t(last);
    } else {
      last = int64_t(v);
    }
  }
  DeviceGuard g(device);
  std::unique_ptr<gnm_pgen> pg(new gnm_pgen);
  pg->device = device;
  pg->variants = m;
  pg->samples = ix.samples;
  pg->file_bytes = pgen_len;
  auto up = [&](const void* src, uint64_t bytes, const char* what) {
    const uint64_t sz = std::max<uint64_t>((bytes + 15) / 16 * 16, 16);
    void* dst = pool_alloc(device, sz, what);
    pg->bufs.push_back(dst);
    pg->device_bytes += sz;
    if (src && bytes) copy_to_device(dst, src, bytes, nullptr);
    return dst;
  };
  PgArgs& a = pg->base;
  a.pgen = static_cast<const uint8_t*>(up(pgen, pgen_len, ".pgen bytes"));
  a.offsets = static_cast<const uint64_t*>(up(ix.offsets.data(), m * 8, ".pgen index"));
  a.lens = static_cast<const uint32_t*>(up(ix.lens.data(), m * 4, ".pgen index"));
  a.types = static_cast<const uint8_t*>(up(ix.types.data(), m, ".pgen index"));
  a.anchor_of = static_cast<const uint32_t*>(up(anchor_of.data(), m * 4, ".pgen index"));
  const uint32_t init_err[2] = {0u, 0xFFFFFFFFu};
  a.err = static_cast<uint32_t*>(up(init_err, 8, ".pgen error word"));
  a.scratch = static_cast<uint8_t*>(up(nullptr, (ix.samples + 3) / 4, ".pgen anchor row"));
  a.n = ix.samples;
  pg->anchor_of = std::move(anchor_of);
  return pg.release();
}

static void pgen_decode_impl(gnm_pgen* pg, uint64_t begin, uint64_t count, uint8_t* d_rows,
                             uint64_t pitch, cudaStream_t s) {
  if (!pg) fail(GNM_ERR_INVALID, "pgen handle is NULL");
  const uint64_t bpv = (pg->samples + 3) / 4;
  if (begin > pg->variants || count > pg->variants - begin)
    fail(GNM_ERR_INVALID, "variant range [" + std::to_string(begin) + ", " +
                              std::to_string(begin + count) + ") exceeds the .pgen's " +
                              std::to_string(pg->variants) + " variants");
  if (count == 0) return;
  if (!d_rows) fail(GNM_ERR_INVALID, "d_rows is NULL");
  if (pitch < bpv || pitch % 16 != 0 || reinterpret_cast<uintptr_t>(d_rows) % 16 != 0)
    fail(GNM_ERR_INVALID, "rows must be 16-byte aligned with a pitch >= ceil(samples/4), "
                          "a multiple of 16");
  PgArgs a = pg->base;
  a.begin = uint32_t(begin);
  a.count = uint32_t(count);
  a.rows = d_rows;
  a.pitch = pitch;
  // the LD records ahead of the range's first non-LD record may anchor before it
  a.extra = kNoAnchor;
  for (uint64_t v = begin; v < begin + count && pg->anchor_of[v] != kNoAnchor; ++v)
    if (pg->anchor_of[v] < begin) {
      a.extra = pg->anchor_of[v];
      break;
    }
  DeviceGuard g(pg->device);
  gnm_pgen_direct<<<a.count + (a.extra != kNoAnchor ? 1u : 0u), kPgThreads, 0, s>>>(a);
  check_cuda(cudaGetLastError(), "pgen decode launch");
  gnm_pgen_ld<<<a.count, kPgThreads, 0, s>>>(a);
  check_cuda(cudaGetLastError(), "pgen LD decode launch");
}

static void pgen_check_impl(gnm_pgen* pg, cudaStream_t s) {
  if (!pg) fail(GNM_ERR_INVALID, "pgen handle is NULL");
  DeviceGuard g(pg->device);
  uint32_t err[2] = {0, 0};
  check_cuda(cudaMemcpyAsync(err, pg->base.err, 8, cudaMemcpyDeviceToHost, s), "pgen error word");
  check_cuda(cudaStreamSynchronize(s), "pgen decode");
  if (err[0])
    fail(GNM_ERR_IO, "malformed .pgen record (variant " + std::to_string(err[1]) +
                         (err[0] & kPgErrPair ? ": bad 1-bit pair code or main-track type"
                                              : ": overruns its length") +
                         ")");
}

}  // namespace gnm

using namespace gnm;

extern "C" {

gnm_status gnm_pgen_dims(const uint8_t* pgen, uint64_t pgen_len, uint64_t* num_variants,
                         uint64_t* num_samples, gnm_error* err) {
  return guarded(err, [&] {
    const PgenIndex ix = parse_pgen(pgen, pgen_len);
    if (num_variants) *num_variants = ix.variants;
    if (num_samples) *num_samples = ix.samples;
  });
}

gnm_status gnm_pgen_open(const uint8_t* pgen, uint64_t pgen_len, int device, gnm_pgen** out,
                         gnm_error* err) {
  return guarded(err, [&] {
    if (!out) fail(GNM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!device_available(device < 0 ? 0 : device)) fail(GNM_DECLINED, "no CUDA device available");
    int dev = device;
    if (dev < 0) check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    *out = pgen_open_impl(pgen, pgen_len, dev);
  });
}

void gnm_pgen_close(gnm_pgen* pg) { delete pg; }

uint64_t gnm_pgen_device_bytes(const gnm_pgen* pg) { return pg ? pg->device_bytes : 0; }

gnm_status gnm_pgen_decode(gnm_pgen* pg, uint64_t variant_begin, uint64_t variant_count,
                           uint8_t* d_rows, uint64_t pitch, void* stream, gnm_error* err) {
  return guarded(err, [&] {
    pgen_decode_impl(pg, variant_begin, variant_count, d_rows, pitch,
                     static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_pgen_check(gnm_pgen* pg, void* stream, gnm_error* err) {
  return guarded(err, [&] { pgen_check_impl(pg, static_cast<cudaStream_t>(stream)); });
}

gnm_status gnm_pgen_decode_device(const uint8_t* pgen, uint64_t pgen_len, int device,
                                  uint8_t* d_rows, uint64_t pitch, void* stream,
                                  gnm_error* err) {
  return guarded(err, [&] {
    if (!device_available(device < 0 ? 0 : device)) fail(GNM_DECLINED, "no CUDA device available");
    int dev = device;
    if (dev < 0) check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    std::unique_ptr<gnm_pgen> pg(pgen_open_impl(pgen, pgen_len, dev));
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    pgen_decode_impl(pg.get(), 0, pg->variants, d_rows, pitch, s);
    pgen_check_impl(pg.get(), s);
  });
}

}  // extern "C"
