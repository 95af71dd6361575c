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
// (variable-width) with or without phase and dosage tracks (dosages fill
// missing hard calls) and, given the variants' ALT counts, multiallelic
// patches (each output row one ALT of a variant; see gnm_pgen_tracks), whose
// main track is type 0 (2-bit),
// 1 (two categories as a bit array + difflist), 2 / 3 (LD-compressed against
// the most recent non-LD record of the same 2^16-variant block; 3 swaps REF and
// ALT homozygotes after the patch) or 4 / 6 / 7 (all hom REF / hom ALT /
// missing + difflist) — shared/adapt_plink2.rs:2237-2257, 2574-2666.  Phase
// tracks follow the main track and do not change hard calls.  Records with
// multiallelic patches are rejected when no ALT counts are given.
//
// Layout of the work: the bijection category -> .bed code lets every step
// run on .bed codes directly.  A decode is two launches over the same
// records, and a third (gnm_pgen_tracks, one CTA per output row) when some
// record carries a multiallelic patch or a dosage track.  Kernel 1 decodes
// the non-LD records, one CTA each: they are few and long (a table pass over
// a whole 2-bit or 1-bit array, or a fill), so eight warps share one.  Kernel 2 decodes the LD-compressed records from
// their anchors' rows, one warp each: they are many, and their work is a
// chain of dependent byte reads, so 64 records per SM stay in flight.  A
// difflist's groups of 64 entries go one per lane: a shuffle scan over the
// group byte lengths places each lane at its group's deltas, and the lane
// walks its base-128 sample-id deltas, four one-byte deltas per step where it
// can.  A lane merges its patches per 32-bit word and writes each word once.
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
constexpr uint32_t kPgWarps = kPgThreads / 32;     // one record per warp
constexpr uint64_t kPgMaxSamples = uint64_t(1) << 31;

enum : uint32_t { kPgErrBounds = 1u, kPgErrPair = 2u, kPgErrPatch = 4u };

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
  uint8_t* scratch;            // anchor rows outside the output: [extra_rows][spitch]
  uint64_t spitch;
  uint32_t extra_rows;         // scratch rows the direct kernel decodes
  // list mode (null in range mode): the variant of output row i (rows count ..
  // count + extra_rows - 1 are scratch rows) and the row holding its anchor
  const uint32_t* vids;
  const uint32_t* arow;
  uint32_t* err;               // [0] error bits, [1] first bad variant (atomicMin)
  uint32_t any_dosage;         // some record carries a dosage track
  const uint32_t* alt_counts;  // [V] ALT alleles per variant (null: every variant biallelic)
  const uint32_t* alt_ords;    // [count] ALT (1-based) of each output row (null: ALT 1)
  uint32_t any_multi;          // some record carries a multiallelic patch to read
  uint32_t ma_smem;            // dynamic shared bytes of the tracks kernel (multiallelic rows)
};

// Row i of a decode: an output row, or a scratch row past the output's end.
__device__ __forceinline__ uint8_t* row_at(const PgArgs& a, uint32_t i) {
  return i < a.count ? a.rows + uint64_t(i) * a.pitch
                     : a.scratch + uint64_t(i - a.count) * a.spitch;
}

// The variant decoded into row i: listed, or the range's (the scratch row of
// a range holds `extra`).
__device__ __forceinline__ uint32_t variant_at(const PgArgs& a, uint32_t i) {
  return a.vids ? a.vids[i] : i < a.count ? a.begin + i : a.extra;
}

__constant__ uint8_t kCatToBed[4] = {0x3, 0x2, 0x0, 0x1};
// 1-bit record pair codes (shared/adapt_plink2.rs:2600-2608): the category of
// a clear bit and of a set bit; -1 = invalid code
__constant__ int8_t kPairLow[16] = {-1, 0, 0, 0, -1, 1, 1, -1, -1, 2, -1, -1, -1, -1, -1, -1};
__constant__ int8_t kPairHigh[16] = {-1, 1, 2, 3, -1, 2, 3, -1, -1, 3, -1, -1, -1, -1, -1, -1};

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

// SWAR REF/ALT swap of sixteen .bed fields: 00 <-> 11, 01 and 10 kept.
__device__ __forceinline__ uint32_t swap_homs(uint32_t x) {
  const uint32_t same = ~(x ^ (x >> 1)) & 0x55555555u;
  return x ^ (same | (same << 1));
}

// Apply the difflist that starts at `cur`; one warp, all lanes call this.
// Layout (shared/adapt_plink2.rs:1920-2040): length (varint); one first sample
// id per group of 64 entries (1-4 bytes by sample count); the byte lengths of
// all but the last group's deltas, minus 63; the 2-bit values; the groups'
// base-128 id deltas.  Groups go 32 at a time, one lane each: a shuffle scan
// over the group byte lengths places each lane at its group's deltas, then
// the lane walks its group.
//
// Sample ids rise strictly (a record that breaks this is malformed), so a
// group owns every 32-bit word of the row between its first and last id
// except those two, which a neighbouring group may share.  A lane merges its
// patches per word in registers and writes each word once: the final value
// computed from `base` (the row before patching: the anchor row of an LD
// record, still in L1 from the copy, with `swap` = type 3's REF/ALT swap
// applied to it and to the patched values; or the row itself) with a plain
// store, or for the two end words and the row's last partial word an
// atomicXor of the patched bits.
//
// `warps` warps may share one difflist: warp `wi` takes the chunks of 32
// groups numbered wi, wi + warps, ...; a strided sum over the group byte
// lengths it skips gives its next chunk's first delta.
__device__ __forceinline__ void warp_difflist(const PgArgs& a, const Rec& r, uint32_t cur,
                                              uint8_t* row, const uint8_t* base, uint32_t v,
                                              bool swap, uint32_t wi = 0, uint32_t warps = 1) {
  const uint32_t lane = threadIdx.x & 31u;
  uint64_t l = 0;
  if (!r.varint(cur, l) || l > a.n) {
    if (lane == 0) flag(a, kPgErrBounds, v);
    return;
  }
  if (l == 0) return;
  const uint32_t len = uint32_t(l);
  const uint32_t groups = (len + 63) / 64;
  const uint32_t wid = a.n <= (1u << 8) ? 1 : a.n <= (1u << 16) ? 2 : a.n <= (1u << 24) ? 3 : 4;
  const uint32_t first_at = cur;
  const uint32_t glen_at = first_at + groups * wid;
  const uint32_t vals_at = glen_at + groups - 1;
  uint32_t deltas = vals_at + (len + 3) / 4;   // the first group's deltas
  if (deltas > r.len) {
    if (lane == 0) flag(a, kPgErrBounds, v);
    return;
  }
  const uint64_t bpv = (a.n + 3) / 4;
  // a word holding bytes past the row's end is only ever xor-patched
  const uint32_t partial_word = bpv % 4 ? uint32_t(bpv / 4) : 0xFFFFFFFFu;
  uint32_t* row32 = reinterpret_cast<uint32_t*>(row);
  const uint32_t* base32 = reinterpret_cast<const uint32_t*>(base);
  auto first_id = [&](uint32_t g) {
    uint64_t id = 0;
    for (uint32_t k = 0; k < wid; ++k) id |= uint64_t(r.p[first_at + g * wid + k]) << (8 * k);
    return id;
  };
  const uint8_t* p = r.p;
  const uint32_t rlen = r.len;
  const uint32_t n32 = uint32_t(a.n);      // samples <= 2^31: ids fit in 32 bits
  // bytes of the deltas of groups [g0, g1), all of which carry a length
  auto skip = [&](uint32_t g0, uint32_t g1) {
    uint32_t s = 0;
    for (uint32_t g = g0 + lane; g < g1; g += 32) s += uint32_t(p[glen_at + g]) + 63u;
#pragma unroll
    for (uint32_t d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, d);
    return s;
  };
  bool bad = false;
  if (wi > 0 && 32 * wi < groups) deltas += skip(0, 32 * wi);
  for (uint32_t c0 = 32 * wi; c0 < groups; c0 += 32 * warps) {
    if (warps > 1 && c0 != 32 * wi) deltas += skip(c0 - 32 * (warps - 1), c0);
    const uint32_t g = c0 + lane;
    // bytes of group g's deltas (all groups but the last carry a length)
    const uint32_t mine = g + 1 < groups ? uint32_t(p[glen_at + g]) + 63u : 0u;
    uint32_t incl = mine;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= d) incl += y;
    }
    uint32_t at = deltas + incl - mine;
    deltas += __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (g >= groups) continue;
    // ids saturate at 2^32 - 1; those >= the sample count are skipped, as
    // the reference skips them
    uint32_t id = uint32_t(min(first_id(g), uint64_t(0xFFFFFFFFu)));
    const uint32_t count = g + 1 < groups ? 64u : len - 64u * (groups - 1);
    const uint32_t start = at;
    const uint8_t* vals = p + vals_at + 16 * g;          // 64 entries = 16 value bytes
    uint32_t cw = 0xFFFFFFFFu;    // word being patched
    uint32_t old = 0;             // its value in `base` (loaded when the word starts)
    uint32_t pm = 0, pv = 0;      // its patched bits and their new values
    bool edge = true;             // the group's first word
    // category -> .bed code as a packed 2-bit table (no divergent lookups):
    // {11, 10, 00, 01}, or with the REF/ALT swap {00, 10, 11, 01}
    const uint32_t code_of = swap ? 0x78u : 0x4Bu;
    // merge the patch of sample `pid` into the word being patched; flush that
    // word when the id moves past it
    auto patch = [&](uint32_t pid, uint32_t val) {
      if (pid >= n32) return;
      const uint32_t code = (code_of >> (2 * val)) & 3u;
      const uint32_t w = pid >> 4;
      const uint32_t sh = 2 * (pid & 15u);
      if (w != cw) {
        if (cw != 0xFFFFFFFFu) {
          const uint32_t o = swap ? swap_homs(old) : old;
          if (edge || cw == partial_word)
            atomicXor(row32 + cw, (o & pm) ^ pv);
          else
            row32[cw] = (o & ~pm) | pv;
          edge = false;
        }
        cw = w;
        old = base32[w];
        pm = pv = 0;
      }
      pm |= 3u << sh;   // ids rise strictly: a field is patched once
      pv |= code << sh;
    };
    patch(id, vals[0] & 3u);   // entry 0: the group's first id
    uint32_t e = 1;
    while (e < count) {
      // four one-byte deltas at once: read as one word (funnel-shifted from
      // aligned words; the record's bytes sit in the file's 16-byte-padded
      // buffer), taken when no byte carries a continuation bit or is zero
      if (e + 4 <= count && at + 4 <= rlen && id < 0xFFFFFE00u) {
        const uintptr_t addr = reinterpret_cast<uintptr_t>(p + at);
        const uint32_t* al = reinterpret_cast<const uint32_t*>(addr & ~uintptr_t(3));
        const uint32_t s8 = uint32_t(addr & 3u) * 8u;
        const uint32_t x = __funnelshift_r(al[0], s8 ? al[1] : 0u, s8);
        if (((x & 0x80808080u) | ((x - 0x01010101u) & ~x & 0x80808080u)) == 0u) {
          // the values of entries e .. e + 3 (a second value byte unless e % 4 == 0)
          const uint32_t lo = vals[e / 4];
          const uint32_t hi = (e & 3u) ? uint32_t(vals[e / 4 + 1]) : 0u;
          const uint32_t vw = (lo | (hi << 8)) >> (2 * (e & 3u));
#pragma unroll
          for (uint32_t k = 0; k < 4; ++k) {
            id += (x >> (8 * k)) & 0xFFu;
            patch(id, (vw >> (2 * k)) & 3u);
          }
          at += 4;
          e += 4;
          continue;
        }
      }
      // one delta, any length; a read past the record gives 0, which ends
      // the walk as a zero delta
      uint32_t d = at < rlen ? p[at] : 0u;
      ++at;
      if (d & 0x80u) {   // multi-byte delta
        uint64_t d64 = d & 0x7Fu;
        uint32_t b, shift = 7;
        do {
          if (at >= rlen || shift > 56) {
            bad = true;
            break;
          }
          b = p[at++];
          d64 |= uint64_t(b & 0x7Fu) << shift;
          shift += 7;
        } while (b & 0x80u);
        if (bad) break;
        d = uint32_t(min(d64, uint64_t(0xFFFFFFFFu)));
      }
      if (d == 0) {
        bad = true;
        break;
      }
      id = id > 0xFFFFFFFFu - d ? 0xFFFFFFFFu : id + d;
      patch(id, (vals[e / 4] >> (2 * (e & 3u))) & 3u);
      ++e;
    }
    if (cw != 0xFFFFFFFFu && !bad) {   // the group's last word
      const uint32_t o = swap ? swap_homs(old) : old;
      atomicXor(row32 + cw, (o & pm) ^ pv);
    }
    if (!bad && g + 1 < groups && (at != start + mine || uint64_t(id) >= first_id(g + 1)))
      bad = true;   // group length mismatch, or ids not rising into the next group
  }
  if (bad) flag(a, kPgErrBounds, v);
}

// Padding fields of the last byte -> 01 (missing), as the reference packs
// them; lane 0, after the warp's writes to the row.
__device__ __forceinline__ void warp_fix_tail(const PgArgs& a, uint8_t* row) {
  __syncwarp();
  const uint32_t rem = uint32_t(a.n % 4);
  if ((threadIdx.x & 31u) == 0 && rem) {
    const uint64_t last = (a.n + 3) / 4 - 1;
    uint32_t b = row[last];
    for (uint32_t k = rem; k < 4; ++k) b = (b & ~(3u << (2 * k))) | (1u << (2 * k));
    row[last] = uint8_t(b);
  }
}

// Padding fields of the last byte -> 01 (missing), after a barrier over the
// CTA's writes to the row.
__device__ __forceinline__ void cta_fix_tail(const PgArgs& a, uint8_t* row) {
  __syncthreads();
  const uint32_t rem = uint32_t(a.n % 4);
  if (threadIdx.x == 0 && rem) {
    const uint64_t last = (a.n + 3) / 4 - 1;
    uint32_t b = row[last];
    for (uint32_t k = rem; k < 4; ++k) b = (b & ~(3u << (2 * k))) | (1u << (2 * k));
    row[last] = uint8_t(b);
  }
}

// One CTA per non-LD record of the range or list (LD-compressed ones return
// at once), plus one per scratch row: anchors outside the output.
// Non-LD records are few and long (whole 2-bit or 1-bit arrays), so all eight
// warps share one: the array pass strided over the CTA, the difflist's
// chunks of 32 groups dealt out across the warps.
__global__ void __launch_bounds__(kPgThreads) gnm_pgen_direct(PgArgs a) {
  __shared__ uint8_t lut[256];     // byte of four PGEN categories -> byte of .bed codes
  __shared__ uint8_t nib[16];      // nibble of four bits -> byte of .bed codes (type 1)
  const uint32_t tid = threadIdx.x;
  const uint32_t v = variant_at(a, blockIdx.x);
  if (a.anchor_of[v] != kNoAnchor) return;
  const Rec r{a.pgen + a.offsets[v], a.lens[v]};
  const uint32_t kind = a.types[v] & 7u;
  uint8_t* row = row_at(a, blockIdx.x);
  const uint64_t bpv = (a.n + 3) / 4;
  const uint64_t words = bpv / 4;
  uint32_t* d32 = reinterpret_cast<uint32_t*>(row);
  uint32_t cur = 0;
  if (kind == 0) {
    if (r.len < bpv) {
      if (tid == 0) flag(a, kPgErrBounds, v);
      return;
    }
    for (uint32_t x = tid; x < 256; x += blockDim.x) {
      uint32_t o = 0;
      for (uint32_t k = 0; k < 4; ++k) o |= uint32_t(kCatToBed[(x >> (2 * k)) & 3u]) << (2 * k);
      lut[x] = uint8_t(o);
    }
    __syncthreads();
    // whole output words from funnel-shifted aligned input words (the record
    // starts at any byte; an aligned word holding a needed byte lies inside
    // the file's 16-byte-padded buffer); four consecutive words per thread and
    // step, five input loads in flight
    const uintptr_t addr = reinterpret_cast<uintptr_t>(r.p);
    const uint32_t* al = reinterpret_cast<const uint32_t*>(addr & ~uintptr_t(3));
    const uint32_t sh = uint32_t(addr & 3u) * 8u;
    for (uint64_t j0 = 4 * uint64_t(tid); j0 < words; j0 += 4 * kPgThreads) {
      uint32_t in[5];
#pragma unroll
      for (uint32_t k = 0; k < 5; ++k) {
        // word j0 + k is needed by output k (k < 4) or by output k - 1's high half
        const bool need = (k < 4 && j0 + k < words) || (sh && k > 0 && j0 + k - 1 < words);
        in[k] = need ? al[j0 + k] : 0u;
      }
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        if (j0 + k >= words) break;
        const uint32_t x = __funnelshift_r(in[k], in[k + 1], sh);
        d32[j0 + k] = uint32_t(lut[x & 255u]) | uint32_t(lut[(x >> 8) & 255u]) << 8 |
                      uint32_t(lut[(x >> 16) & 255u]) << 16 | uint32_t(lut[x >> 24]) << 24;
      }
    }
    for (uint64_t j = 4 * words + tid; j < bpv; j += blockDim.x) row[j] = lut[r.p[j]];
    cta_fix_tail(a, row);
    return;
  }
  if (kind == 1) {
    // pair code -> (low, high) categories; bit set = high
    uint32_t pc = 0;
    const bool okb = r.byte(0, pc);
    const int low = okb && pc < 16 ? kPairLow[pc] : -1;
    const int high = okb && pc < 16 ? kPairHigh[pc] : -1;
    if (!okb || low < 0) {
      if (tid == 0) flag(a, kPgErrPair, v);
      return;
    }
    const uint32_t nb = uint32_t((a.n + 7) / 8);
    if (r.len < 1 + nb) {
      if (tid == 0) flag(a, kPgErrBounds, v);
      return;
    }
    if (tid < 16) {
      uint32_t o = 0;
      for (uint32_t k = 0; k < 4; ++k)
        o |= uint32_t(kCatToBed[((tid >> k) & 1u) ? high : low]) << (2 * k);
      nib[tid] = uint8_t(o);
    }
    __syncthreads();
    const uint8_t* bits = r.p + 1;
    for (uint64_t j = tid; j < words; j += blockDim.x) {
      const uint32_t b0 = bits[2 * j], b1 = bits[2 * j + 1];
      d32[j] = uint32_t(nib[b0 & 15u]) | uint32_t(nib[b0 >> 4]) << 8 |
               uint32_t(nib[b1 & 15u]) << 16 | uint32_t(nib[b1 >> 4]) << 24;
    }
    for (uint64_t j = 4 * words + tid; j < bpv; j += blockDim.x)
      row[j] = nib[(bits[j / 2] >> (4 * (j % 2))) & 15u];
    cur = 1 + nb;
  } else if (kind == 4 || kind == 6 || kind == 7) {
    const uint32_t byte = kCatToBed[kind == 4 ? 0 : kind == 6 ? 2 : 3] * 0x55u;
    const uint32_t w = byte * 0x01010101u;
    const uint4 q = make_uint4(w, w, w, w);
    const uint64_t vecs = bpv / 16;
    for (uint64_t j = tid; j < vecs; j += blockDim.x) reinterpret_cast<uint4*>(row)[j] = q;
    for (uint64_t j = 16 * vecs + tid; j < bpv; j += blockDim.x) row[j] = uint8_t(byte);
  } else {
    if (tid == 0) flag(a, kPgErrPair, v);
    return;
  }
  __syncthreads();   // the row is complete before its words are patched
  warp_difflist(a, r, cur, row, row, v, false, tid / 32, kPgWarps);
  cta_fix_tail(a, row);
}

// One warp per LD-compressed record of the range or list (others return at
// once; eight CTAs, 64 warps, per SM): copy the anchor row (16-byte vectors; type 3 swaps REF and ALT homozygotes
// on the way), then patch it with the record's difflist.  The anchor row is an
// output row, or a scratch row when it is outside the output.
__global__ void __launch_bounds__(kPgThreads, 8) gnm_pgen_ld(PgArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t wi = uint64_t(blockIdx.x) * kPgWarps + threadIdx.x / 32;
  if (wi >= a.count) return;
  const uint32_t v = variant_at(a, uint32_t(wi));
  const uint32_t anchor = a.anchor_of[v];
  if (anchor == kNoAnchor) return;
  const Rec r{a.pgen + a.offsets[v], a.lens[v]};
  const bool swap = (a.types[v] & 7u) == 3u;
  uint8_t* row = a.rows + wi * a.pitch;
  const uint32_t ar = a.arow ? a.arow[wi] : anchor >= a.begin ? anchor - a.begin : a.count;
  const uint8_t* src = row_at(a, ar);
  const uint64_t bpv = (a.n + 3) / 4;
  const uint64_t vecs = bpv / 16;
  const uint4* s16 = reinterpret_cast<const uint4*>(src);
  uint4* d16 = reinterpret_cast<uint4*>(row);
  // four 16-byte loads in flight per lane before their stores
  uint64_t j = lane;
  for (; j + 96 < vecs; j += 128) {
    uint4 q[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = s16[j + 32 * k];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (swap) {
        q[k].x = swap_homs(q[k].x);
        q[k].y = swap_homs(q[k].y);
        q[k].z = swap_homs(q[k].z);
        q[k].w = swap_homs(q[k].w);
      }
      d16[j + 32 * k] = q[k];
    }
  }
  for (; j < vecs; j += 32) {
    uint4 q = s16[j];
    if (swap) {
      q.x = swap_homs(q.x);
      q.y = swap_homs(q.y);
      q.z = swap_homs(q.z);
      q.w = swap_homs(q.w);
    }
    d16[j] = q;
  }
  for (uint64_t b = 16 * vecs + lane; b < bpv; b += 32)
    row[b] = uint8_t(swap ? swap_homs(src[b]) : src[b]);
  __syncwarp();
  warp_difflist(a, r, 0, row, src, v, swap);
  warp_fix_tail(a, row);
}


// ---- dosage tracks ---------------------------------------------------------------
// A biallelic record may carry, after its main track (and its phase track,
// vrtype bit 4), a dosage track (bits 5-6, shared/adapt_plink2.rs:2416-2520):
// u16 ALT dosages (16384 per allele copy, 65535 = none) for a sample list
// (bit 5: an id-only difflist), for every sample (bit 6), or for the samples
// of a presence bit array (bits 5 + 6); bit 7 adds a phased-dosage track
// after it, which does not change hard calls.  Where the hard call is missing,
// the dosage becomes the nearest whole allele count if it lies within 0.10 of
// it (f32 arithmetic, :3211-3255), else the call stays missing.  Hard calls are
// never overridden; samples are diploid (the .pvar/.psam that give the
// reference its ploidy are not read here).  The overlay runs after both decode
// kernels, on whole rows, so LD records still read their anchors' raw calls.

// .bed code of a u16 diploid ALT dosage, or 01 (missing) when none applies.
__device__ __forceinline__ uint32_t dosage_code(uint32_t v) {
  if (v == 65535u) return 1u;
  const float ds = float(v) * (1.0f / 32768.0f) * 2.0f;
  // nearest of 0, 1, 2 (first wins a tie, as the reference scans them in order)
  const float d0 = fabsf(ds), d1 = fabsf(ds - 1.0f), d2 = fabsf(ds - 2.0f);
  uint32_t best = 0;
  float bd = d0;
  if (d1 < bd) { best = 1; bd = d1; }
  if (d2 < bd) { best = 2; bd = d2; }
  if (!(bd <= 0.10f)) return 1u;
  return best == 2 ? 0u : (best == 1 ? 2u : 3u);   // ALT count 2 -> 00, 1 -> 10, 0 -> 11
}

// Sum over the 256 threads of the CTA (every thread calls it).
__device__ __forceinline__ uint32_t cta_sum(uint32_t x, uint32_t* sh) {
#pragma unroll
  for (uint32_t d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, d);
  __syncthreads();
  if ((threadIdx.x & 31u) == 0) sh[threadIdx.x >> 5] = x;
  __syncthreads();
  uint32_t t = 0;
#pragma unroll
  for (uint32_t w = 0; w < kPgWarps; ++w) t += sh[w];
  return t;
}

// Exclusive prefix over the 256 threads of the CTA; `total` gets the sum.
__device__ __forceinline__ uint32_t cta_exclusive(uint32_t x, uint32_t* sh, uint32_t& total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = x;
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d) incl += y;
  }
  __syncthreads();
  if (lane == 31) sh[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  total = 0;
#pragma unroll
  for (uint32_t w = 0; w < kPgWarps; ++w) {
    if (w < warp) before += sh[w];
    total += sh[w];
  }
  return before + incl - x;
}

// Byte just past a difflist at `cur` (ids_only: no 2-bit values, the dosage
// track's sample list).  Every thread returns it; false = the list overruns
// the record.  Group byte lengths are summed by the CTA, the last group's
// deltas walked by thread 0.
__device__ bool cta_difflist_end(const Rec& r, uint32_t cur, uint64_t n, bool ids_only,
                                 uint32_t* sh, uint32_t& end) {
  uint64_t l = 0;
  bool ok = r.varint(cur, l) && l <= n;
  if (!ok) return false;
  if (l == 0) {
    end = cur;
    return true;
  }
  const uint32_t len = uint32_t(l);
  const uint32_t groups = (len + 63) / 64;
  const uint32_t wid = n <= (1u << 8) ? 1 : n <= (1u << 16) ? 2 : n <= (1u << 24) ? 3 : 4;
  const uint64_t glen_at = uint64_t(cur) + uint64_t(groups) * wid;
  const uint64_t deltas = glen_at + groups - 1 + (ids_only ? 0 : (len + 3) / 4);
  if (deltas > r.len) return false;
  uint32_t part = 0;
  for (uint32_t g = threadIdx.x; g + 1 < groups; g += blockDim.x)
    part += uint32_t(r.p[glen_at + g]) + 63u;
  const uint32_t before_last = cta_sum(part, sh);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t at = uint32_t(min(deltas + before_last, uint64_t(0xFFFFFFFFu)));
    const uint32_t count = len - 64u * (groups - 1);
    bool good = deltas + before_last <= r.len;
    for (uint32_t e = 1; good && e < count; ++e) {
      uint64_t d;
      good = r.varint(at, d);
    }
    sh[kPgWarps] = good ? at : 0xFFFFFFFFu;
  }
  __syncthreads();
  end = sh[kPgWarps];
  __syncthreads();
  return end != 0xFFFFFFFFu;
}

// Walk an id-only difflist that starts at `cur` (already checked whole by
// cta_difflist_end): fn(e, id) for every entry e whose sample id is below n,
// called by the thread that owns the entry's group of 64.  Returns false on
// ids that do not rise or a group byte length that does not match (the same
// on every thread).
template <class F>
__device__ bool cta_walk_ids(const Rec& r, uint32_t cur, uint64_t n, uint32_t* sh, F fn) {
  uint64_t l = 0;
  uint32_t c2 = cur;
  r.varint(c2, l);
  if (l == 0) return true;
  const uint32_t len = uint32_t(l);
  const uint32_t groups = (len + 63) / 64;
  const uint32_t wid = n <= (1u << 8) ? 1 : n <= (1u << 16) ? 2 : n <= (1u << 24) ? 3 : 4;
  const uint32_t first_at = c2;
  const uint32_t glen_at = first_at + groups * wid;
  const uint32_t deltas0 = glen_at + groups - 1;
  auto first_id = [&](uint32_t g) {
    uint64_t id = 0;
    for (uint32_t k = 0; k < wid; ++k) id |= uint64_t(r.p[first_at + g * wid + k]) << (8 * k);
    return id;
  };
  uint32_t base = deltas0;   // first delta byte of this chunk's first group
  bool broken = false;
  for (uint32_t g0 = 0; g0 < groups; g0 += blockDim.x) {
    const uint32_t g = g0 + threadIdx.x;
    const uint32_t mine = g + 1 < groups ? uint32_t(r.p[glen_at + g]) + 63u : 0u;
    uint32_t total = 0;
    uint32_t at = base + cta_exclusive(g < groups ? mine : 0u, sh, total);
    if (g < groups && !broken) {
      const uint32_t count = g + 1 < groups ? 64u : len - 64u * (groups - 1);
      const uint32_t start = at;
      uint64_t id = first_id(g);
      for (uint32_t e = 0; e < count; ++e) {
        if (e > 0) {
          uint64_t d = 0;
          if (!r.varint(at, d) || d == 0) {
            broken = true;
            break;
          }
          id += d;
        }
        if (id < n) fn(64u * g + e, id);
      }
      if (!broken && g + 1 < groups && (at != start + mine || id >= first_id(g + 1)))
        broken = true;   // group length mismatch, or ids not rising into the next group
    }
    base += total;
  }
  return !__syncthreads_or(broken);
}

// ---- multiallelic patches --------------------------------------------------------
// A record of a variant with two or more ALT alleles may carry, right after
// its main track, a patch (vrtype bit 3, shared/adapt_plink2.rs:2704-2881):
// one format byte (low nibble: hets, high nibble: hom-ALT category; 0 = a bit
// array over that category's samples in order, 1 = an id-only difflist, 15 =
// no patch), then per category the patched samples and their values: a het's
// ALT minus 2 in a fixed width set by the ALT count, or a hom-ALT-category
// pair's two ALTs minus 1 (two ALTs: one flag bit per sample, set = ALT 2 /
// ALT 2, clear = ALT 1 / ALT 2).  Unpatched hets are REF / ALT 1 and unpatched
// hom-ALTs ALT 1 / ALT 1.  A decoded row holds the copies of one ALT j as .bed
// codes, the reference's virtual .bed splitting the variant into one row per
// ALT.

__device__ __forceinline__ uint32_t het_alt_width(uint32_t ac) {
  return ac == 2 ? 0u : ac == 3 ? 1u : ac <= 5 ? 2u : ac <= 17 ? 4u : ac <= 257 ? 8u : 16u;
}
__device__ __forceinline__ uint32_t homalt_width(uint32_t ac) {
  return ac <= 4 ? 2u : ac <= 16 ? 4u : ac <= 256 ? 8u : 16u;
}
// .bed code of `c` copies of the row's ALT
__device__ __forceinline__ uint32_t copies_code(uint32_t c) {
  return c == 2 ? 0u : (c == 1 ? 2u : 3u);
}
// Field e of a run of w-bit little-endian fields (1 <= w <= 16) at byte `at`;
// the caller checked that the run lies inside the record.
__device__ __forceinline__ uint32_t packed_field(const uint8_t* p, uint64_t at, uint32_t w,
                                                 uint64_t e) {
  const uint64_t bit = e * w;
  const uint8_t* b = p + at + (bit >> 3);
  const uint32_t s = uint32_t(bit & 7u);
  uint32_t x = b[0];
  if (s + w > 8) x |= uint32_t(b[1]) << 8;
  if (s + w > 16) x |= uint32_t(b[2]) << 16;
  return (x >> s) & ((1u << w) - 1u);
}
// Bits [b0, b0 + cnt) (cnt <= 16) of a bit array of `nbytes` bytes at `at`.
__device__ __forceinline__ uint32_t bits_at(const uint8_t* p, uint64_t at, uint64_t nbytes,
                                            uint64_t b0, uint32_t cnt) {
  if (cnt == 0) return 0u;
  const uint64_t byte0 = b0 >> 3;
  const uint32_t s = uint32_t(b0 & 7u);
  uint32_t x = 0;
  for (uint32_t k = 0; k < 3 && 8 * k < s + cnt; ++k)
    if (byte0 + k < nbytes) x |= uint32_t(p[at + byte0 + k]) << (8 * k);
  return (x >> s) & ((1u << cnt) - 1u);
}

struct MaSection {
  uint32_t fmt;       // 0 bit array, 1 id difflist, 15 none
  uint32_t sel_at;    // the bit array or difflist
  uint64_t sel_bytes; // bit array bytes
  uint32_t k;         // patched samples
  uint32_t vals_at;   // their values
};

// Parse one category's section at `cur` (every thread, same result); false =
// it overruns the record.  `members`: the category's sample count.
__device__ bool ma_section(const Rec& r, uint32_t& cur, uint32_t fmt, uint64_t n,
                           uint32_t members, bool het, uint32_t ac, uint32_t* sh, MaSection& s) {
  s.fmt = fmt;
  s.k = 0;
  s.sel_at = s.vals_at = cur;
  s.sel_bytes = 0;
  if (fmt == 15) return true;
  if (fmt == 0) {
    s.sel_bytes = (uint64_t(members) + 7) / 8;
    if (uint64_t(cur) + s.sel_bytes > r.len) return false;
    uint32_t part = 0;
    for (uint64_t b = threadIdx.x; b < s.sel_bytes; b += blockDim.x) {
      uint32_t byte = r.p[cur + b];
      const uint64_t left = uint64_t(members) - 8 * b;
      if (left < 8) byte &= (1u << left) - 1u;
      part += __popc(byte);
    }
    s.k = cta_sum(part, sh);
    cur += uint32_t(s.sel_bytes);
  } else {
    uint32_t end = 0;
    if (!cta_difflist_end(r, cur, n, true, sh, end)) return false;
    uint64_t l = 0;
    uint32_t c2 = cur;
    r.varint(c2, l);
    s.k = uint32_t(l);
    cur = end;
  }
  s.vals_at = cur;
  const uint64_t vb = het ? (uint64_t(s.k) * het_alt_width(ac) + 7) / 8
                          : ac == 2 ? (uint64_t(s.k) + 7) / 8
                                    : (2 * uint64_t(s.k) * homalt_width(ac) + 7) / 8;
  if (uint64_t(cur) + vb > r.len) return false;
  cur += uint32_t(vb);
  return true;
}

// ALT of the het in patch entry e.
__device__ __forceinline__ uint32_t ma_het_alt(const Rec& r, const MaSection& s, uint32_t ac,
                                               uint64_t e) {
  const uint32_t w = het_alt_width(ac);
  return w == 0 ? 2u : packed_field(r.p, s.vals_at, w, e) + 2u;
}
// Copies of ALT j in the hom-ALT-category pair of patch entry e.
__device__ __forceinline__ uint32_t ma_hom_copies(const Rec& r, const MaSection& s, uint32_t ac,
                                                  uint64_t e, uint32_t j) {
  if (ac == 2) {
    const bool two = (r.p[s.vals_at + (e >> 3)] >> (e & 7u)) & 1u;   // ALT 2 / ALT 2
    return two ? (j == 2 ? 2u : 0u) : (j <= 2 ? 1u : 0u);
  }
  const uint32_t w = homalt_width(ac);
  const uint32_t lo = packed_field(r.p, s.vals_at, w, 2 * e) + 1u;
  const uint32_t hi = packed_field(r.p, s.vals_at, w, 2 * e + 1) + 1u;
  return uint32_t(lo == j) + uint32_t(hi == j);
}

// Project a multiallelic record's row onto ALT j.  The row holds the main
// track's codes; `orig` (shared, one word per 16 samples) gets a copy of
// them, which the patch entries are checked against.  `cur` is at the patch
// and ends past it.  Returns 0, or the error bit to set.
__device__ uint32_t ma_project(const Rec& r, uint32_t& cur, uint64_t n, uint32_t ac, uint32_t j,
                               uint32_t* row32, uint64_t words, uint32_t* orig, uint32_t* sh) {
  auto valid = [&](uint64_t w) {   // 2-bit fields of real samples in word w
    const uint64_t s0 = 16 * w;
    return s0 + 16 <= n ? 0xFFFFFFFFu : (n > s0 ? (1u << (2 * (n - s0))) - 1u : 0u);
  };
  uint32_t hets = 0, homs = 0;
  for (uint64_t w = threadIdx.x; w < words; w += blockDim.x) {
    const uint32_t x = row32[w];
    orig[w] = x;
    hets += __popc((x >> 1) & ~x & 0x55555555u & valid(w));    // code 10
    homs += __popc(~x & ~(x >> 1) & 0x55555555u & valid(w));   // code 00
  }
  hets = cta_sum(hets, sh);
  homs = cta_sum(homs, sh);
  if (cur >= r.len) return kPgErrBounds;
  const uint32_t fmt = r.p[cur++];
  const uint32_t f1 = fmt & 15u, f2 = fmt >> 4;
  MaSection s1, s2;
  if (f1 != 0 && f1 != 1 && f1 != 15) return kPgErrPatch;
  if (!ma_section(r, cur, f1, n, hets, true, ac, sh, s1)) return kPgErrBounds;
  if (f2 != 0 && f2 != 1 && f2 != 15) return kPgErrPatch;
  if (!ma_section(r, cur, f2, n, homs, false, ac, sh, s2)) return kPgErrBounds;
  const uint32_t het_dflt = j == 1 ? 2u : 3u;                // REF / ALT 1
  const uint32_t hom_dflt = copies_code(j == 1 ? 2u : 0u);   // ALT 1 / ALT 1

  // Pass 1, a word of 16 samples per thread: unpatched calls and the patches
  // given as bit arrays (ranks within the category by CTA scans).
  uint32_t base_h = 0, base_a = 0, base_hv = 0, base_av = 0;
  for (uint64_t w0 = 0; w0 < words; w0 += blockDim.x) {
    const uint64_t w = w0 + threadIdx.x;
    uint32_t x = 0, hm = 0, am = 0;
    if (w < words) {
      x = orig[w];
      hm = (x >> 1) & ~x & 0x55555555u & valid(w);
      am = ~x & ~(x >> 1) & 0x55555555u & valid(w);
    }
    uint32_t tot = 0;
    const uint32_t hr = base_h + cta_exclusive(__popc(hm), sh, tot);   // rank of the word's first het
    base_h += tot;
    const uint32_t ar = base_a + cta_exclusive(__popc(am), sh, tot);
    base_a += tot;
    const uint32_t hb = s1.fmt == 0 && w < words
                            ? bits_at(r.p, s1.sel_at, s1.sel_bytes, hr, __popc(hm)) : 0u;
    const uint32_t ab = s2.fmt == 0 && w < words
                            ? bits_at(r.p, s2.sel_at, s2.sel_bytes, ar, __popc(am)) : 0u;
    const uint32_t hv = base_hv + cta_exclusive(__popc(hb), sh, tot);   // value index of its first patch
    base_hv += tot;
    const uint32_t av = base_av + cta_exclusive(__popc(ab), sh, tot);
    base_av += tot;
    if (w < words) {
      uint32_t y = x, hi = 0, ai = 0, hs = 0, as = 0;
      for (uint32_t k = 0; k < 16; ++k) {
        const uint32_t f = 2 * k;
        uint32_t code;
        if ((hm >> f) & 1u) {
          code = het_dflt;
          if ((hb >> hi) & 1u) code = ma_het_alt(r, s1, ac, hv + hs++) == j ? 2u : 3u;
          ++hi;
        } else if ((am >> f) & 1u) {
          code = hom_dflt;
          if ((ab >> ai) & 1u) code = copies_code(ma_hom_copies(r, s2, ac, av + as++, j));
          ++ai;
        } else {
          continue;
        }
        y = (y & ~(3u << f)) | (code << f);
      }
      if (y != x) row32[w] = y;
    }
  }
  __syncthreads();
  // Pass 2: patches given as sample lists; a listed sample of the right
  // category flips its field from the pass-1 code to the patched one.
  bool ok = true;
  if (s1.fmt == 1)
    ok = cta_walk_ids(r, s1.sel_at, n, sh, [&](uint32_t e, uint64_t id) {
      const uint32_t wd = uint32_t(id >> 4), f = 2 * uint32_t(id & 15u);
      if (((orig[wd] >> f) & 3u) != 2u) return;
      const uint32_t code = ma_het_alt(r, s1, ac, e) == j ? 2u : 3u;
      if (code != het_dflt) atomicXor(row32 + wd, (code ^ het_dflt) << f);
    });
  if (ok && s2.fmt == 1)
    ok = cta_walk_ids(r, s2.sel_at, n, sh, [&](uint32_t e, uint64_t id) {
      const uint32_t wd = uint32_t(id >> 4), f = 2 * uint32_t(id & 15u);
      if (((orig[wd] >> f) & 3u) != 0u) return;
      const uint32_t code = copies_code(ma_hom_copies(r, s2, ac, e, j));
      if (code != hom_dflt) atomicXor(row32 + wd, (code ^ hom_dflt) << f);
    });
  __syncthreads();
  return ok ? 0u : kPgErrBounds;
}

// One CTA per output row; rows whose record has neither a multiallelic patch
// (for a variant with two or more ALTs) nor a dosage track return at once.
// Runs after gnm_pgen_direct and gnm_pgen_ld have written the rows, so LD
// records read their anchors' raw calls.  Dynamic shared memory: one word per
// 16 samples when the decode holds multiallelic rows.
__global__ void __launch_bounds__(kPgThreads) gnm_pgen_tracks(PgArgs a) {
  extern __shared__ uint32_t s_orig[];
  __shared__ uint32_t sh[kPgWarps + 2];
  const uint32_t i = blockIdx.x;
  if (i >= a.count) return;
  const uint32_t v = variant_at(a, i);
  const uint32_t t = a.types[v];
  const uint32_t ac = a.alt_counts ? a.alt_counts[v] : 1u;
  const uint32_t j = a.alt_ords ? a.alt_ords[i] : 1u;
  // shared/adapt_plink2.rs:2348-2362: the patch is read only for a variant
  // with two or more ALTs (otherwise the record reads as biallelic and the
  // patch bytes are not skipped); only ALT 1 rows take dosages (:2420)
  const bool multi = (t & 0x08u) && ac >= 2;
  if (!multi && !(t & 0x60u)) return;
  const bool apply_dosage = ac <= 1 || j == 1;
  const Rec r{a.pgen + a.offsets[v], a.lens[v]};
  const uint64_t n = a.n;
  const uint64_t bpv = (n + 3) / 4;
  uint8_t* row = a.rows + uint64_t(i) * a.pitch;
  uint32_t* row32 = reinterpret_cast<uint32_t*>(row);
  const uint64_t words = (bpv + 3) / 4;
  auto bad = [&]() {
    if (threadIdx.x == 0) flag(a, kPgErrBounds, v);
  };

  // ---- the main track's end ----
  const uint32_t kind = t & 7u;
  uint32_t cur = 0;
  if (kind == 0) {
    cur = uint32_t(bpv);
  } else {
    const uint32_t start = kind == 1 ? uint32_t(1 + (n + 7) / 8) : 0u;
    if (!cta_difflist_end(r, start, n, false, sh, cur)) return bad();
  }
  if (cur > r.len) return bad();

  // het calls of the main track (.bed code 10), which size the phase track
  uint32_t h = 0;
  if (t & 0x10u) {
    uint32_t hets = 0;
    for (uint64_t w = threadIdx.x; w < words; w += blockDim.x) {
      uint32_t x = row32[w];
      const uint64_t b0 = 4 * w;
      if (b0 + 4 > bpv) x &= (1u << (8 * (bpv - b0))) - 1u;   // bytes past the row
      hets += __popc((x >> 1) & ~x & 0x55555555u);
    }
    h = cta_sum(hets, sh);
  }

  // ---- the multiallelic patch ----
  if (multi) {
    const uint32_t e = ma_project(r, cur, n, ac, j, row32, words, s_orig, sh);
    if (e) {
      if (threadIdx.x == 0) flag(a, e, v);
      return;
    }
  }

  // ---- the phase track: one flag bit, per-het presence bits padded to a
  // byte when the flag is set, one bit per phased het ----
  if (t & 0x10u) {
    if (cur >= r.len) return bad();
    uint64_t bits = 1 + uint64_t(h);
    if (r.p[cur] & 1u) {
      // presence bits 1 .. h, then one phase bit per present het
      uint32_t present = 0;
      const uint64_t nbytes = (1 + uint64_t(h) + 7) / 8;
      if (cur + nbytes > r.len) return bad();
      for (uint64_t b = threadIdx.x; b < nbytes; b += blockDim.x) {
        uint32_t byte = r.p[cur + b];
        if (b == 0) byte &= ~1u;
        const uint64_t hi = 1 + uint64_t(h) - 8 * b;   // bits of this byte in range
        if (hi < 8) byte &= (1u << hi) - 1u;
        present += __popc(byte);
      }
      const uint32_t phased = cta_sum(present, sh);
      bits = (bits + 7) / 8 * 8 + phased;
    }
    const uint64_t next = cur + (bits + 7) / 8;
    if (next > r.len) return bad();
    cur = uint32_t(next);
  }

  // ---- the dosage track (read for its bounds on every row, applied on rows
  // of ALT 1); row words are read through L2 (a multiallelic patch may have
  // just updated them with atomics) ----
  if (!(t & 0x60u)) return;
  const bool b5 = t & 0x20u, b6 = t & 0x40u;
  if (b6 && !b5) {
    // dense: every sample's value
    if (uint64_t(cur) + 2 * n > r.len) return bad();
    if (!apply_dosage) return;
    const uint8_t* vals = r.p + cur;
    for (uint64_t w = threadIdx.x; w < words; w += blockDim.x) {
      const uint32_t x = __ldcg(row32 + w);
      uint32_t y = x;
#pragma unroll 4
      for (uint32_t k = 0; k < 16; ++k) {
        const uint64_t smp = 16 * w + k;
        if (smp >= n) break;
        if (((x >> (2 * k)) & 3u) != 1u) continue;
        const uint32_t dv = uint32_t(vals[2 * smp]) | (uint32_t(vals[2 * smp + 1]) << 8);
        y = (y & ~(3u << (2 * k))) | (dosage_code(dv) << (2 * k));
      }
      if (y != x) row32[w] = y;
    }
    return;
  }
  if (b5 && b6) {
    // presence bit array, then the values of the present samples in order
    const uint64_t pbytes = (n + 7) / 8;
    if (uint64_t(cur) + pbytes > r.len) return bad();
    const uint8_t* pres = r.p + cur;
    const uint64_t vals_at = uint64_t(cur) + pbytes;
    uint32_t base = 0;   // present samples before this chunk of words
    for (uint64_t w0 = 0; w0 < words; w0 += blockDim.x) {
      const uint64_t w = w0 + threadIdx.x;
      uint32_t mask = 0;   // presence bits of the word's 16 samples
      if (w < words) {
        for (uint32_t k = 0; k < 16; ++k) {
          const uint64_t smp = 16 * w + k;
          if (smp < n && ((pres[smp >> 3] >> (smp & 7)) & 1u)) mask |= 1u << k;
        }
      }
      uint32_t total = 0;
      const uint32_t before = base + cta_exclusive(__popc(mask), sh, total);
      if (apply_dosage && w < words && mask) {
        const uint32_t x = __ldcg(row32 + w);
        uint32_t y = x, rank = 0;
        for (uint32_t k = 0; k < 16; ++k) {
          if (!((mask >> k) & 1u)) continue;
          const uint64_t at = vals_at + 2 * uint64_t(before + rank);
          ++rank;
          if (((x >> (2 * k)) & 3u) != 1u) continue;
          if (at + 2 > r.len) {
            flag(a, kPgErrBounds, v);
            break;
          }
          const uint32_t dv = uint32_t(r.p[at]) | (uint32_t(r.p[at + 1]) << 8);
          y = (y & ~(3u << (2 * k))) | (dosage_code(dv) << (2 * k));
        }
        if (y != x) row32[w] = y;
      }
      base += total;
    }
    if (threadIdx.x == 0 && vals_at + 2 * uint64_t(base) > r.len) flag(a, kPgErrBounds, v);
    return;
  }
  // b5 alone: an id-only difflist, then one value per listed sample
  uint32_t list_end = 0;
  if (!cta_difflist_end(r, cur, n, true, sh, list_end)) return bad();
  uint64_t l = 0;
  uint32_t c2 = cur;
  r.varint(c2, l);
  if (uint64_t(list_end) + 2 * l > r.len) return bad();
  const bool ok = cta_walk_ids(r, cur, n, sh, [&](uint32_t e, uint64_t id) {
    if (!apply_dosage) return;
    const uint32_t w = uint32_t(id >> 4), sh2 = 2 * uint32_t(id & 15u);
    if (((__ldcg(row32 + w) >> sh2) & 3u) != 1u) return;
    const uint64_t vat = uint64_t(list_end) + 2 * uint64_t(e);
    const uint32_t dv = uint32_t(r.p[vat]) | (uint32_t(r.p[vat + 1]) << 8);
    const uint32_t code = dosage_code(dv);
    // the field is 01: xor it to the new code (ids rise, so no other thread
    // writes this field; fields of one word commute)
    if (code != 1u) atomicXor(row32 + w, (1u ^ code) << sh2);
  });
  if (!ok) bad();
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
PgenIndex parse_pgen(const uint8_t* d, uint64_t len, bool have_alts = false) {
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
    // records start after the 12 header bytes, one more byte and (reference
    // flag mode 3) one reference flag bit per variant, where the reference's
    // reader puts them (shared/adapt_plink2.rs:2048-2057, asserted by its
    // test at :3826-3866)
    const uint64_t rec = (ix.samples + 3) / 4;
    const uint64_t base = 13 + (((d[11] >> 6) & 3) == 3 ? (m + 7) / 8 : 0);
    for (uint64_t v = 0; v < m; ++v) {
      ix.offsets[v] = base + v * rec;
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
    if ((ix.types[v] & 0x08u) && !have_alts)
      fail(GNM_ERR_INVALID, "variant " + std::to_string(v) +
                                ": a multiallelic record needs the variants' ALT counts");
    if ((ix.types[v] & 0x80u) && !(ix.types[v] & 0x60u))
      fail(GNM_ERR_IO, "variant " + std::to_string(v) +
                           ": phased dosage track without a dosage track");
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
  std::vector<uint32_t> anchor_of;   // host copy: which anchors a decode needs
  std::vector<uint32_t> alt_counts;  // host copy (empty: every variant biallelic)
  std::vector<void*> bufs;
  gnm::PgArgs base{};
  // list-mode buffers, grown on demand (device and host copies)
  uint8_t* scratch = nullptr;
  uint64_t scratch_rows = 0;
  uint32_t* d_list = nullptr;        // [vids | arow]
  uint64_t list_cap = 0;
  std::vector<uint32_t> h_list;
  ~gnm_pgen() {
    // decodes in flight on any stream may still read the buffers
    gnm::DeviceGuard g(device);
    cudaDeviceSynchronize();
    for (void* x : bufs) gnm::pool_free(x);
    gnm::pool_free(scratch);
    gnm::pool_free(d_list);
  }
};

namespace gnm {

// Largest dynamic shared memory of a tracks CTA (one word per 16 samples of
// a multiallelic row), under the 227 KB per-block limit.
constexpr uint64_t kPgMaSmemMax = 220 * 1024;

gnm_pgen* pgen_open_impl(const uint8_t* pgen, uint64_t pgen_len, int device,
                         const uint32_t* alt_counts) {
  PgenIndex ix = parse_pgen(pgen, pgen_len, alt_counts != nullptr);
  const uint64_t m = ix.variants;
  bool any_multi = false;
  if (alt_counts) {
    for (uint64_t v = 0; v < m; ++v) {
      if (alt_counts[v] < 1 || alt_counts[v] > 65535)
        fail(GNM_ERR_INVALID, "variant " + std::to_string(v) + ": ALT count " +
                                  std::to_string(alt_counts[v]) + " is outside 1..65535");
      any_multi = any_multi || ((ix.types[v] & 0x08u) && alt_counts[v] >= 2);
    }
  }
  const uint64_t ma_smem = any_multi ? ((ix.samples + 3) / 4 + 3) / 4 * 4 : 0;
  if (ma_smem > kPgMaSmemMax)
    fail(GNM_ERR_INVALID, "multiallelic records of more than " +
                              std::to_string(kPgMaSmemMax / 4 * 16) + " samples");
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
  a.any_dosage = 0u;
  for (uint64_t v = 0; v < m && !a.any_dosage; ++v) a.any_dosage = (ix.types[v] & 0x60u) ? 1u : 0u;
  a.alt_counts = alt_counts ? static_cast<const uint32_t*>(up(alt_counts, m * 4, ".pgen ALT counts"))
                            : nullptr;
  a.alt_ords = nullptr;
  a.any_multi = any_multi ? 1u : 0u;
  a.ma_smem = uint32_t(ma_smem);
  pg->alt_counts.assign(alt_counts ? alt_counts : nullptr, alt_counts ? alt_counts + m : nullptr);
  const uint32_t init_err[2] = {0u, 0xFFFFFFFFu};
  a.err = static_cast<uint32_t*>(up(init_err, 8, ".pgen error word"));
  a.spitch = ((ix.samples + 3) / 4 + 15) / 16 * 16;
  pg->scratch = static_cast<uint8_t*>(pool_alloc(device, a.spitch, ".pgen anchor rows"));
  pg->scratch_rows = 1;
  pg->device_bytes += a.spitch;
  a.scratch = pg->scratch;
  a.n = ix.samples;
  pg->anchor_of = std::move(anchor_of);
  return pg.release();
}

// Grow a handle buffer; work in flight may read the old one, so the device
// is synchronised before it is freed (growth is rare: the first large list).
template <class T>
static void grow(gnm_pgen* pg, T*& buf, uint64_t& cap, uint64_t need, uint64_t unit,
                 const char* what) {
  if (need <= cap) return;
  check_cuda(cudaDeviceSynchronize(), what);
  pool_free(buf);
  pg->device_bytes -= cap * unit;
  buf = nullptr;
  cap = 0;
  buf = static_cast<T*>(pool_alloc(pg->device, need * unit, what));
  cap = need;
  pg->device_bytes += need * unit;
}

static void check_rows(const gnm_pgen* pg, const uint8_t* d_rows, uint64_t pitch) {
  const uint64_t bpv = (pg->samples + 3) / 4;
  if (!d_rows) fail(GNM_ERR_INVALID, "d_rows is NULL");
  if (pitch < bpv || pitch % 16 != 0 || reinterpret_cast<uintptr_t>(d_rows) % 16 != 0)
    fail(GNM_ERR_INVALID, "rows must be 16-byte aligned with a pitch >= ceil(samples/4), "
                          "a multiple of 16");
}

static void launch_decode(const PgArgs& a, cudaStream_t s) {
  gnm_pgen_direct<<<a.count + a.extra_rows, kPgThreads, 0, s>>>(a);
  check_cuda(cudaGetLastError(), "pgen decode launch");
  gnm_pgen_ld<<<uint32_t((uint64_t(a.count) + kPgWarps - 1) / kPgWarps), kPgThreads, 0, s>>>(a);
  check_cuda(cudaGetLastError(), "pgen LD decode launch");
  if (a.any_dosage || a.any_multi) {   // patches and dosages, on the finished rows
    if (a.ma_smem > 48 * 1024)
      check_cuda(raise_smem_limit(reinterpret_cast<const void*>(gnm_pgen_tracks), int(a.ma_smem)),
                 "pgen tracks shared memory");
    gnm_pgen_tracks<<<a.count, kPgThreads, a.any_multi ? a.ma_smem : 0u, s>>>(a);
    check_cuda(cudaGetLastError(), "pgen tracks launch");
  }
}

// Decode the listed variants (any order) into consecutive rows.  An LD
// record whose anchor is not listed reads it from a scratch row the same
// launch decodes; every such anchor is decoded once.
void pgen_decode_list_impl(gnm_pgen* pg, const uint64_t* list, uint64_t count,
                                  uint8_t* d_rows, uint64_t pitch, cudaStream_t s,
                                  const uint32_t* alt_ords) {
  if (!pg) fail(GNM_ERR_INVALID, "pgen handle is NULL");
  if (count == 0) return;
  if (!list) fail(GNM_ERR_INVALID, "variant list is NULL");
  if (alt_ords) {
    for (uint64_t i = 0; i < count; ++i) {
      if (list[i] >= pg->variants) break;   // reported below
      const uint32_t ac = pg->alt_counts.empty() ? 1u : pg->alt_counts[list[i]];
      if (alt_ords[i] < 1 || alt_ords[i] > ac)
        fail(GNM_ERR_INVALID, "row " + std::to_string(i) + ": ALT " + std::to_string(alt_ords[i]) +
                                  " of variant " + std::to_string(list[i]) + ", which has " +
                                  std::to_string(ac) + " ALT allele(s)");
    }
  }
  check_rows(pg, d_rows, pitch);
  if (count > 0x3FFFFFFFull) fail(GNM_ERR_INVALID, "more than 2^30 - 1 listed variants");
  std::vector<std::pair<uint32_t, uint32_t>> sorted(count);   // (variant, row)
  for (uint64_t i = 0; i < count; ++i) {
    if (list[i] >= pg->variants)
      fail(GNM_ERR_INVALID, "listed variant " + std::to_string(list[i]) + " is past the .pgen's " +
                                std::to_string(pg->variants) + " variants");
    sorted[i] = {uint32_t(list[i]), uint32_t(i)};
  }
  std::sort(sorted.begin(), sorted.end());
  std::vector<uint32_t>& h = pg->h_list;
  h.assign(2 * count, 0u);   // vids (+ scratch variants appended), then arow
  std::vector<uint32_t> extra;
  std::vector<std::pair<uint32_t, uint32_t>> slot;             // (anchor, scratch row)
  for (uint64_t i = 0; i < count; ++i) {
    const uint32_t a = pg->anchor_of[list[i]];
    h[i] = uint32_t(list[i]);
    if (a == kNoAnchor) continue;
    auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(a, 0u));
    if (it != sorted.end() && it->first == a) {
      h[count + i] = it->second;
    } else {
      auto sl = std::lower_bound(slot.begin(), slot.end(), std::make_pair(a, 0u));
      if (sl == slot.end() || sl->first != a) {
        sl = slot.insert(sl, {a, uint32_t(extra.size())});
        extra.push_back(a);
      }
      h[count + i] = uint32_t(count) + sl->second;
    }
  }
  // layout on the device: vids [count + extra], arow [count], ALTs [count]
  std::vector<uint32_t> dev(2 * count + extra.size() + (alt_ords ? count : 0));
  std::copy(h.begin(), h.begin() + count, dev.begin());
  std::copy(extra.begin(), extra.end(), dev.begin() + count);
  std::copy(h.begin() + count, h.end(), dev.begin() + count + extra.size());
  if (alt_ords) std::copy(alt_ords, alt_ords + count, dev.begin() + 2 * count + extra.size());
  pg->h_list.swap(dev);   // kept alive by the handle until the next call
  DeviceGuard g(pg->device);
  grow(pg, pg->d_list, pg->list_cap, pg->h_list.size(), sizeof(uint32_t), ".pgen variant list");
  grow(pg, pg->scratch, pg->scratch_rows, std::max<uint64_t>(1, extra.size()), pg->base.spitch,
       ".pgen anchor rows");
  check_cuda(cudaMemcpyAsync(pg->d_list, pg->h_list.data(), pg->h_list.size() * 4,
                             cudaMemcpyHostToDevice, s),
             "upload .pgen variant list");
  PgArgs a = pg->base;
  a.scratch = pg->scratch;
  a.count = uint32_t(count);
  a.rows = d_rows;
  a.pitch = pitch;
  a.extra_rows = uint32_t(extra.size());
  a.vids = pg->d_list;
  a.arow = pg->d_list + count + extra.size();
  a.alt_ords = alt_ords ? pg->d_list + 2 * count + extra.size() : nullptr;
  launch_decode(a, s);
}

static void pgen_decode_impl(gnm_pgen* pg, uint64_t begin, uint64_t count, uint8_t* d_rows,
                             uint64_t pitch, cudaStream_t s) {
  if (!pg) fail(GNM_ERR_INVALID, "pgen handle is NULL");
  if (begin > pg->variants || count > pg->variants - begin)
    fail(GNM_ERR_INVALID, "variant range [" + std::to_string(begin) + ", " +
                              std::to_string(begin + count) + ") exceeds the .pgen's " +
                              std::to_string(pg->variants) + " variants");
  if (count == 0) return;
  check_rows(pg, d_rows, pitch);
  PgArgs a = pg->base;
  a.scratch = pg->scratch;
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
  a.extra_rows = a.extra != kNoAnchor ? 1u : 0u;
  DeviceGuard g(pg->device);
  launch_decode(a, s);
}

uint64_t pgen_samples(const gnm_pgen* pg) { return pg->samples; }
uint64_t pgen_variants(const gnm_pgen* pg) { return pg->variants; }

void pgen_check_impl(gnm_pgen* pg, cudaStream_t s) {
  if (!pg) fail(GNM_ERR_INVALID, "pgen handle is NULL");
  DeviceGuard g(pg->device);
  uint32_t err[2] = {0, 0};
  check_cuda(cudaMemcpyAsync(err, pg->base.err, 8, cudaMemcpyDeviceToHost, s), "pgen error word");
  check_cuda(cudaStreamSynchronize(s), "pgen decode");
  if (err[0])
    fail(GNM_ERR_IO, "malformed .pgen record (variant " + std::to_string(err[1]) +
                         (err[0] & kPgErrPair    ? ": bad 1-bit pair code or main-track type"
                          : err[0] & kPgErrPatch ? ": unsupported multiallelic patch format"
                                                 : ": overruns its length") +
                         ")");
}

}  // namespace gnm

using namespace gnm;

extern "C" {

gnm_status gnm_pgen_dims(const uint8_t* pgen, uint64_t pgen_len, uint64_t* num_variants,
                         uint64_t* num_samples, gnm_error* err) {
  return guarded(err, [&] {
    // the counts only: multiallelic records are checked when the file is
    // opened, with or without ALT counts
    const PgenIndex ix = parse_pgen(pgen, pgen_len, true);
    if (num_variants) *num_variants = ix.variants;
    if (num_samples) *num_samples = ix.samples;
  });
}

gnm_status gnm_pgen_open(const uint8_t* pgen, uint64_t pgen_len, int device, gnm_pgen** out,
                         gnm_error* err) {
  return guarded(err, [&] {
    if (!out) fail(GNM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    const int dev = resolve_device(device);
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

gnm_status gnm_pgen_decode_list(gnm_pgen* pg, const uint64_t* variants, uint64_t count,
                                uint8_t* d_rows, uint64_t pitch, void* stream, gnm_error* err) {
  return guarded(err, [&] {
    pgen_decode_list_impl(pg, variants, count, d_rows, pitch, static_cast<cudaStream_t>(stream));
  });
}

gnm_status gnm_pgen_open_alleles(const uint8_t* pgen, uint64_t pgen_len,
                                 const uint32_t* alt_counts, int device, gnm_pgen** out,
                                 gnm_error* err) {
  return guarded(err, [&] {
    if (!out) fail(GNM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!alt_counts) fail(GNM_ERR_INVALID, "alt_counts is NULL");
    const int dev = resolve_device(device);
    *out = pgen_open_impl(pgen, pgen_len, dev, alt_counts);
  });
}

gnm_status gnm_pgen_decode_alleles(gnm_pgen* pg, const uint64_t* variants,
                                   const uint32_t* alt_ords, uint64_t count, uint8_t* d_rows,
                                   uint64_t pitch, void* stream, gnm_error* err) {
  return guarded(err, [&] {
    if (count && !alt_ords) fail(GNM_ERR_INVALID, "alt_ords is NULL");
    pgen_decode_list_impl(pg, variants, count, d_rows, pitch, static_cast<cudaStream_t>(stream),
                          alt_ords);
  });
}

gnm_status gnm_pgen_check(gnm_pgen* pg, void* stream, gnm_error* err) {
  return guarded(err, [&] { pgen_check_impl(pg, static_cast<cudaStream_t>(stream)); });
}

gnm_status gnm_pgen_decode_device(const uint8_t* pgen, uint64_t pgen_len, int device,
                                  uint8_t* d_rows, uint64_t pitch, void* stream,
                                  gnm_error* err) {
  return guarded(err, [&] {
    const int dev = resolve_device(device);
    std::unique_ptr<gnm_pgen> pg(pgen_open_impl(pgen, pgen_len, dev));
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    pgen_decode_impl(pg.get(), 0, pg->variants, d_rows, pitch, s);
    pgen_check_impl(pg.get(), s);
  });
}

}  // extern "C"
