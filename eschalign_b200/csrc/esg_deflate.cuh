// BGZF block compression on the device: one warp per BGZF block, DEFLATE
// (RFC 1951) with one dynamic-Huffman block per BGZF block.
//
// The BGZF writer of the BAM stage cuts the record stream into blocks of at
// most 0xff00 bytes and deflates each on its own; the host cores at zlib's
// level 6 spend about 11 core-seconds per million 150-nt records on it.
// Blocks are independent, so here each one is a CTA of one warp:
//   1. each lane runs a greedy LZ77 over its 2040-byte stripe of the block
//      (a private 2048-entry table of the last position per 4-byte hash, primed
//      with the 512 bytes before the stripe, matches clipped at the stripe's
//      end) and writes its tokens to global scratch, counting the literal /
//      length and distance symbols in shared memory;
//   2. lane 0 builds the length-limited Huffman codes (two-queue Huffman on
//      the sorted frequencies, lengths folded to 15 bits by moving leaves
//      down until Kraft's sum is one) and the block header (code lengths
//      run-length coded with symbols 16/17/18, RFC 1951 section 3.2.7);
//   3. each lane sums its tokens' bits, a warp scan gives every lane its
//      bit offset, and the lanes write their bits into the block's output
//      slot (whole words with plain stores, the two shared edge words with
//      atomicOr).
// A block whose code would not be smaller than a stored block is reported
// as such (length kStored) and the host writes it stored.  The output is a
// valid DEFLATE stream that any inflater reads; it is not byte-identical to
// zlib's (the records it holds are).
//
// Every function below except the kernel is __host__ __device__: the host
// build runs the same steps lane by lane (esg_bgzf_deflate_host), which
// is how the CPU tests check them against zlib's inflate.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __CUDACC__
#define ESG_DHD __host__ __device__
#else
#define ESG_DHD
#endif

namespace esg_deflate {

constexpr uint32_t kBlockIn = 0xff00;                 // input bytes per BGZF block
constexpr uint32_t kLanes = 32;
constexpr uint32_t kLaneBytes = kBlockIn / kLanes;     // 2040: one stripe per lane
constexpr uint32_t kSlotBytes = 65536;                 // output slot per block
constexpr uint32_t kHashBits = 11;
constexpr uint32_t kHashSize = 1u << kHashBits;        // per-lane table entries
constexpr uint16_t kEmpty = 0xffff;
constexpr uint32_t kMinMatch = 4;
constexpr uint32_t kMaxMatch = 258;
constexpr uint32_t kLookback = 512;                    // bytes before a stripe primed
constexpr uint32_t kStored = 0xffffffffu;              // "write this block stored"
constexpr uint32_t kNumLit = 286;                      // literal / length symbols
constexpr uint32_t kNumDist = 30;
constexpr uint32_t kNumCl = 19;                        // code-length symbols
constexpr uint32_t kMaxSyms = 288;
constexpr uint32_t kTokensPerBlock = kLanes * kLaneBytes;
constexpr uint32_t kMatchFlag = 0x80000000u;

// Shared state of one block.  The per-lane hash tables and the staged input
// dominate (128 KiB + 64 KiB): one CTA per SM.
struct BlockState {
  uint8_t in[kBlockIn];
  uint16_t table[kLanes * kHashSize];
  uint32_t lit_freq[kMaxSyms];
  uint32_t dist_freq[32];
  uint32_t cl_freq[kNumCl + 1];
  uint8_t lit_len[kMaxSyms];
  uint8_t dist_len[32];
  uint8_t cl_len[kNumCl + 1];
  uint16_t lit_code[kMaxSyms];
  uint16_t dist_code[32];
  uint16_t cl_code[kNumCl + 1];
  // the header's run-length items: symbol (5 bits) << 8 | extra value
  uint16_t items[kNumLit + kNumDist];
  uint32_t n_items;
  uint32_t n_lit, n_dist, n_cl;
  uint32_t header_bits;
  uint32_t lane_bits[kLanes];
  // Huffman scratch (lane 0)
  uint32_t h_weight[2 * kMaxSyms];
  uint16_t h_parent[2 * kMaxSyms];
  uint16_t h_sorted[kMaxSyms];
};

ESG_DHD inline uint32_t clz32(uint32_t x) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__clz((int)x);
#else
  return x ? (uint32_t)__builtin_clz(x) : 32u;
#endif
}

ESG_DHD inline uint32_t hash4(const uint8_t* p) {
  const uint32_t x = (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 |
                     (uint32_t)p[3] << 24;
  return (x * 2654435761u) >> (32 - kHashBits);
}

// Length L (3..258) -> symbol 257..285, extra bit count and value
// (RFC 1951 section 3.2.5).
ESG_DHD inline void length_symbol(uint32_t L, uint32_t& sym, uint32_t& nx, uint32_t& xv) {
  const uint32_t l = L - 3;
  if (l < 8) {
    sym = 257 + l;
    nx = 0;
    xv = 0;
  } else if (L == 258) {
    sym = 285;
    nx = 0;
    xv = 0;
  } else {
    const uint32_t nb = 31 - clz32(l);  // 3..7
    sym = 257 + 4 * (nb - 1) + ((l >> (nb - 2)) & 3);
    nx = nb - 2;
    xv = l & ((1u << nx) - 1);
  }
}

// Distance D (1..32768) -> symbol 0..29, extra bit count and value.
ESG_DHD inline void distance_symbol(uint32_t D, uint32_t& sym, uint32_t& nx, uint32_t& xv) {
  const uint32_t d = D - 1;
  if (d < 4) {
    sym = d;
    nx = 0;
    xv = 0;
  } else {
    const uint32_t nb = 31 - clz32(d);  // 2..14
    sym = 2 * nb + ((d >> (nb - 1)) & 1);
    nx = nb - 1;
    xv = d & ((1u << nx) - 1);
  }
}

// Counters: shared-memory atomics on the device, plain adds on the host.
ESG_DHD inline void count(uint32_t* c) {
#ifdef __CUDA_ARCH__
  atomicAdd(c, 1u);
#else
  ++*c;
#endif
}

// Step 1 for one lane: greedy LZ77 over the lane's stripe of the block
// `d[0, n)`; tokens (a byte, or kMatchFlag | (L - 3) << 15 | (D - 1)) go to
// tok[k * stride].  Returns the token count (at most kLaneBytes).
ESG_DHD inline uint32_t lz_stripe(const uint8_t* d, uint32_t n, uint32_t lane, uint16_t* tab,
                                  uint32_t* tok, uint32_t stride, uint32_t* lit_freq,
                                  uint32_t* dist_freq) {
  const uint32_t s = lane * kLaneBytes;
  if (s >= n) return 0;
  const uint32_t e = s + kLaneBytes < n ? s + kLaneBytes : n;
  for (uint32_t i = 0; i < kHashSize; ++i) tab[i] = kEmpty;
  for (uint32_t p = s > kLookback ? s - kLookback : 0; p < s; ++p)
    if (p + 4 <= n) tab[hash4(d + p)] = (uint16_t)p;
  uint32_t nt = 0, p = s;
  while (p < e) {
    uint32_t L = 0, c = kEmpty;
    if (p + kMinMatch <= e) {
      const uint32_t h = hash4(d + p);
      c = tab[h];
      tab[h] = (uint16_t)p;
      if (c != kEmpty) {  // c < p: every entry is an earlier position
        const uint32_t lim = e - p < kMaxMatch ? e - p : kMaxMatch;
        while (L < lim && d[c + L] == d[p + L]) ++L;
        if (L < kMinMatch) L = 0;
      }
    }
    if (L) {
      const uint32_t D = p - c;
      tok[(size_t)nt++ * stride] = kMatchFlag | (L - 3) << 15 | (D - 1);
      uint32_t sym, nx, xv;
      length_symbol(L, sym, nx, xv);
      count(lit_freq + sym);
      distance_symbol(D, sym, nx, xv);
      count(dist_freq + sym);
      for (uint32_t q = p + 1; q < p + L; ++q)
        if (q + 4 <= n) tab[hash4(d + q)] = (uint16_t)q;
      p += L;
    } else {
      tok[(size_t)nt++ * stride] = d[p];
      count(lit_freq + d[p]);
      ++p;
    }
  }
  return nt;
}

// Code lengths for freq[0, n) of at most `limit` bits.  Symbols with a
// frequency get a length; if fewer than two have one, the first unused
// symbols get frequency 1, so the code is always complete.  Scratch in S.
ESG_DHD inline void huffman_lengths(const uint32_t* freq, uint32_t n, uint32_t limit,
                                    uint8_t* len, BlockState& S) {
  uint32_t* w = S.h_weight;
  uint16_t* par = S.h_parent;
  uint16_t* sorted = S.h_sorted;
  uint32_t m = 0;
  for (uint32_t i = 0; i < n; ++i) {
    len[i] = 0;
    if (freq[i]) sorted[m++] = (uint16_t)i;
  }
  for (uint32_t i = 0; m < 2 && i < n; ++i)
    if (!freq[i]) {
      // keep `sorted` in symbol order: insert i where it belongs
      uint32_t k = m++;
      while (k > 0 && sorted[k - 1] > i) {
        sorted[k] = sorted[k - 1];
        --k;
      }
      sorted[k] = (uint16_t)i;
    }
  auto weight = [&](uint32_t sym) { return freq[sym] ? freq[sym] : 1u; };
  // insertion sort on (weight, symbol); symbols arrive in symbol order
  for (uint32_t i = 1; i < m; ++i) {
    const uint16_t x = sorted[i];
    const uint32_t wx = weight(x);
    uint32_t k = i;
    while (k > 0 && weight(sorted[k - 1]) > wx) {
      sorted[k] = sorted[k - 1];
      --k;
    }
    sorted[k] = x;
  }
  // two-queue Huffman: leaves 0..m-1 by weight, internal nodes m..2m-2 are
  // made in nondecreasing weight order
  for (uint32_t i = 0; i < m; ++i) w[i] = weight(sorted[i]);
  uint32_t li = 0, ii = m, nx = m;
  for (uint32_t k = 0; k + 1 < m; ++k) {
    uint32_t pick[2];
    for (int t = 0; t < 2; ++t) {
      if (li < m && (ii >= nx || w[li] <= w[ii]))
        pick[t] = li++;
      else
        pick[t] = ii++;
    }
    w[nx] = w[pick[0]] + w[pick[1]];
    par[pick[0]] = par[pick[1]] = (uint16_t)nx;
    ++nx;
  }
  // depths (reuse w): the root is 2m-2, parents come after their children
  uint32_t bl_count[32] = {};
  w[2 * m - 2] = 0;
  for (int32_t i = (int32_t)(2 * m) - 3; i >= 0; --i) w[i] = w[par[i]] + 1;
  uint32_t maxd = 0;
  for (uint32_t i = 0; i < m; ++i) {
    const uint32_t dpt = w[i] < 31 ? w[i] : 31;
    ++bl_count[dpt];
    if (dpt > maxd) maxd = dpt;
  }
  if (maxd > limit) {
    // fold lengths above the limit into it, then move leaves one level
    // down until Kraft's sum is exactly one
    for (uint32_t L = limit + 1; L <= maxd; ++L) {
      bl_count[limit] += bl_count[L];
      bl_count[L] = 0;
    }
    uint64_t total = 0;
    for (uint32_t L = 1; L <= limit; ++L) total += (uint64_t)bl_count[L] << (limit - L);
    while (total > (1ull << limit)) {
      --bl_count[limit];
      for (uint32_t L = limit - 1; L > 0; --L)
        if (bl_count[L]) {
          --bl_count[L];
          bl_count[L + 1] += 2;
          break;
        }
      --total;
    }
    maxd = limit;
  }
  // the lightest leaves take the longest codes
  uint32_t at = 0;
  for (uint32_t L = maxd; L >= 1; --L)
    for (uint32_t c = 0; c < bl_count[L]; ++c) len[sorted[at++]] = (uint8_t)L;
}

// Canonical codes (RFC 1951 section 3.2.2), bit-reversed for an LSB-first
// stream.
ESG_DHD inline void canonical_codes(const uint8_t* len, uint32_t n, uint16_t* code) {
  uint32_t bl_count[16] = {}, next[16] = {};
  for (uint32_t i = 0; i < n; ++i) ++bl_count[len[i]];
  bl_count[0] = 0;
  uint32_t c = 0;
  for (uint32_t L = 1; L < 16; ++L) {
    c = (c + bl_count[L - 1]) << 1;
    next[L] = c;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t L = len[i];
    code[i] = 0;
    if (!L) continue;
    uint32_t v = next[L]++, r = 0;
    for (uint32_t b = 0; b < L; ++b) r |= ((v >> b) & 1u) << (L - 1 - b);
    code[i] = (uint16_t)r;
  }
}

// Order in which the code-length code's lengths are sent.
ESG_DHD inline uint32_t cl_order(uint32_t i) {
  const uint8_t o[kNumCl] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
  return o[i];
}

ESG_DHD inline uint32_t cl_extra_bits(uint32_t sym) {
  return sym == 16 ? 2u : sym == 17 ? 3u : sym == 18 ? 7u : 0u;
}

// Step 2 (lane 0): the codes and the header's items; S.header_bits is the
// header's length in bits (BFINAL, BTYPE, HLIT, HDIST, HCLEN, the
// code-length code, the items).
ESG_DHD inline void build_codes(BlockState& S) {
  S.lit_freq[256] += 1;  // end of block
  huffman_lengths(S.lit_freq, kNumLit, 15, S.lit_len, S);
  huffman_lengths(S.dist_freq, kNumDist, 15, S.dist_len, S);
  canonical_codes(S.lit_len, kNumLit, S.lit_code);
  canonical_codes(S.dist_len, kNumDist, S.dist_code);
  uint32_t nl = kNumLit, nd = kNumDist;
  while (nl > 257 && !S.lit_len[nl - 1]) --nl;
  while (nd > 1 && !S.dist_len[nd - 1]) --nd;
  S.n_lit = nl;
  S.n_dist = nd;
  // run-length items over the lengths of lit 0..nl-1 then dist 0..nd-1
  auto at = [&](uint32_t i) -> uint32_t { return i < nl ? S.lit_len[i] : S.dist_len[i - nl]; };
  const uint32_t total = nl + nd;
  for (uint32_t i = 0; i < kNumCl; ++i) S.cl_freq[i] = 0;
  uint32_t ni = 0;
  auto item = [&](uint32_t sym, uint32_t xv) {
    S.items[ni++] = (uint16_t)(sym << 8 | xv);
    ++S.cl_freq[sym];
  };
  for (uint32_t i = 0; i < total;) {
    const uint32_t cur = at(i);
    uint32_t run = 1;
    while (i + run < total && at(i + run) == cur) ++run;
    i += run;
    if (cur == 0) {
      while (run >= 11) {
        const uint32_t r = run < 138 ? run : 138;
        item(18, r - 11);
        run -= r;
      }
      if (run >= 3) {
        item(17, run - 3);
        run = 0;
      }
      while (run--) item(0, 0);
    } else {
      item(cur, 0);
      --run;
      while (run >= 3) {
        const uint32_t r = run < 6 ? run : 6;
        item(16, r - 3);
        run -= r;
      }
      while (run--) item(cur, 0);
    }
  }
  S.n_items = ni;
  huffman_lengths(S.cl_freq, kNumCl, 7, S.cl_len, S);
  canonical_codes(S.cl_len, kNumCl, S.cl_code);
  uint32_t ncl = kNumCl;
  while (ncl > 4 && !S.cl_len[cl_order(ncl - 1)]) --ncl;
  S.n_cl = ncl;
  uint32_t bits = 3 + 5 + 5 + 4 + 3 * ncl;
  for (uint32_t k = 0; k < ni; ++k) {
    const uint32_t sym = S.items[k] >> 8;
    bits += S.cl_len[sym] + cl_extra_bits(sym);
  }
  S.header_bits = bits;
}

ESG_DHD inline uint32_t token_bits(const BlockState& S, uint32_t t) {
  if (!(t & kMatchFlag)) return S.lit_len[t];
  uint32_t sym, nx, xv;
  length_symbol(((t >> 15) & 0xff) + 3, sym, nx, xv);
  uint32_t b = S.lit_len[sym] + nx;
  distance_symbol((t & 0x7fff) + 1, sym, nx, xv);
  return b + S.dist_len[sym] + nx;
}

// LSB-first bit writer over 32-bit words: the first word and the last
// (partial) word of a lane's range may be shared with its neighbours and
// are OR-ed in; the words in between are the lane's alone.
struct BitSink {
  uint32_t* out;
  uint64_t acc;
  uint32_t nacc;
  uint32_t word;
  bool first;
  ESG_DHD BitSink(uint32_t* o, uint64_t bit) : out(o), acc(0), nacc((uint32_t)(bit & 31)),
                                               word((uint32_t)(bit >> 5)), first(true) {}
  ESG_DHD void shared_or(uint32_t v) {
#ifdef __CUDA_ARCH__
    if (v) atomicOr(out + word, v);
#else
    out[word] |= v;
#endif
  }
  ESG_DHD void put(uint32_t v, uint32_t nb) {  // nb <= 32, v < 2^nb
    if (!nb) return;
    acc |= (uint64_t)v << nacc;
    nacc += nb;
    while (nacc >= 32) {
      const uint32_t x = (uint32_t)acc;
      if (first)
        shared_or(x);
      else
        out[word] = x;
      first = false;
      acc >>= 32;
      nacc -= 32;
      ++word;
    }
  }
  ESG_DHD void finish() {
    if (nacc) shared_or((uint32_t)acc);
  }
};

// The dynamic block header (lane 0's stream starts with it).
ESG_DHD inline void put_header(const BlockState& S, BitSink& o) {
  o.put(1, 1);  // BFINAL
  o.put(2, 2);  // BTYPE = 10: dynamic Huffman
  o.put(S.n_lit - 257, 5);
  o.put(S.n_dist - 1, 5);
  o.put(S.n_cl - 4, 4);
  for (uint32_t i = 0; i < S.n_cl; ++i) o.put(S.cl_len[cl_order(i)], 3);
  for (uint32_t k = 0; k < S.n_items; ++k) {
    const uint32_t sym = S.items[k] >> 8, xv = S.items[k] & 0xff;
    o.put(S.cl_code[sym], S.cl_len[sym]);
    o.put(xv, cl_extra_bits(sym));
  }
}

ESG_DHD inline void put_token(const BlockState& S, BitSink& o, uint32_t t) {
  if (!(t & kMatchFlag)) {
    o.put(S.lit_code[t], S.lit_len[t]);
    return;
  }
  uint32_t sym, nx, xv;
  length_symbol(((t >> 15) & 0xff) + 3, sym, nx, xv);
  o.put(S.lit_code[sym], S.lit_len[sym]);
  o.put(xv, nx);
  distance_symbol((t & 0x7fff) + 1, sym, nx, xv);
  o.put(S.dist_code[sym], S.dist_len[sym]);
  o.put(xv, nx);
}

}  // namespace esg_deflate

namespace esg_deflate {

// The steps of the kernel below, lane by lane on the host: `out` (kSlotBytes
// bytes, 4-byte aligned) receives the DEFLATE stream of d[0, n); returns its
// length in bytes, or kStored.  Used by the CPU tests of the steps.
inline uint32_t deflate_block_host(const uint8_t* d, uint32_t n, uint8_t* out, BlockState& S,
                                   uint32_t* tokens /* kTokensPerBlock */) {
  for (uint32_t i = 0; i < n && i < kBlockIn; ++i) S.in[i] = d[i];
  for (uint32_t i = 0; i < kMaxSyms; ++i) S.lit_freq[i] = 0;
  for (uint32_t i = 0; i < 32; ++i) S.dist_freq[i] = 0;
  uint32_t nt[kLanes], bits[kLanes];
  for (uint32_t l = 0; l < kLanes; ++l)
    nt[l] = lz_stripe(S.in, n, l, S.table + l * kHashSize, tokens + l, kLanes, S.lit_freq,
                      S.dist_freq);
  build_codes(S);
  uint32_t total = 0;
  for (uint32_t l = 0; l < kLanes; ++l) {
    bits[l] = l == 0 ? S.header_bits : 0;
    for (uint32_t k = 0; k < nt[l]; ++k) bits[l] += token_bits(S, tokens[(size_t)k * kLanes + l]);
    if (l == kLanes - 1) bits[l] += S.lit_len[256];
    total += bits[l];
  }
  const uint32_t bytes = (total + 7) / 8;
  if (bytes > n + 5) return kStored;
  uint32_t* o = reinterpret_cast<uint32_t*>(out);
  for (uint32_t i = 0; i < (total + 31) / 32; ++i) o[i] = 0;
  uint32_t start = 0;
  for (uint32_t l = 0; l < kLanes; ++l) {
    BitSink sink(o, start);
    if (l == 0) put_header(S, sink);
    for (uint32_t k = 0; k < nt[l]; ++k) put_token(S, sink, tokens[(size_t)k * kLanes + l]);
    if (l == kLanes - 1) sink.put(S.lit_code[256], S.lit_len[256]);
    sink.finish();
    start += bits[l];
  }
  return bytes;
}

#ifdef __CUDACC__
// One CTA of one warp per BGZF block b: in[b * kBlockIn, ...) of n_in bytes
// in all -> out[b * kSlotBytes / 4, ...) and out_len[b] (bytes, or
// kStored).  tokens: kTokensPerBlock words of scratch per block.  Dynamic
// shared memory: sizeof(BlockState).
__global__ void __launch_bounds__(32) k_bgzf_deflate(const uint8_t* __restrict__ in,
                                                      uint64_t n_in, uint32_t* __restrict__ tokens,
                                                      uint32_t* __restrict__ out,
                                                      uint32_t* __restrict__ out_len) {
  extern __shared__ __align__(16) uint8_t smem[];
  BlockState& S = *reinterpret_cast<BlockState*>(smem);
  const uint32_t b = blockIdx.x, lane = threadIdx.x;
  const uint64_t base = (uint64_t)b * kBlockIn;
  if (base >= n_in) return;
  const uint32_t n = (uint32_t)(n_in - base < kBlockIn ? n_in - base : kBlockIn);
  // stage the block (kBlockIn is a multiple of 16, so every block starts
  // 16-byte aligned when `in` does)
  const uint4* src = reinterpret_cast<const uint4*>(in + base);
  uint4* dst = reinterpret_cast<uint4*>(S.in);
  for (uint32_t i = lane; i < n / 16; i += kLanes) dst[i] = src[i];
  for (uint32_t i = n / 16 * 16 + lane; i < n; i += kLanes) S.in[i] = in[base + i];
  for (uint32_t i = lane; i < kMaxSyms; i += kLanes) S.lit_freq[i] = 0;
  S.dist_freq[lane] = 0;
  __syncwarp();
  uint32_t* tok = tokens + (size_t)b * kTokensPerBlock + lane;
  const uint32_t nt = lz_stripe(S.in, n, lane, S.table + lane * kHashSize, tok, kLanes,
                                S.lit_freq, S.dist_freq);
  __syncwarp();
  if (lane == 0) build_codes(S);
  __syncwarp();
  uint32_t bits = lane == 0 ? S.header_bits : 0;
  for (uint32_t k = 0; k < nt; ++k) bits += token_bits(S, tok[(size_t)k * kLanes]);
  if (lane == kLanes - 1) bits += S.lit_len[256];
  uint32_t incl = bits;
  for (uint32_t dd = 1; dd < kLanes; dd <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, dd);
    if (lane >= dd) incl += v;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, kLanes - 1);
  const uint32_t bytes = (total + 7) / 8;
  if (bytes > n + 5) {  // a stored block is no larger
    if (lane == 0) out_len[b] = kStored;
    return;
  }
  // bytes <= n + 5 <= kBlockIn + 5 < kSlotBytes: every word below is in the slot
  uint32_t* o = out + (size_t)b * (kSlotBytes / 4);
  for (uint32_t i = lane; i < (total + 31) / 32; i += kLanes) o[i] = 0;
  __syncwarp();
  BitSink sink(o, incl - bits);
  if (lane == 0) put_header(S, sink);
  for (uint32_t k = 0; k < nt; ++k) put_token(S, sink, tok[(size_t)k * kLanes]);
  if (lane == kLanes - 1) sink.put(S.lit_code[256], S.lit_len[256]);
  sink.finish();
  if (lane == 0) out_len[b] = bytes;
}
#endif

}  // namespace esg_deflate
