// esg_bam.cu -- BAM input and output around the mapping stage (host code).
//
// The CLI's I/O stage (crates/eschalign-cli/src/align.rs):
//   * reading: read_batches (align.rs:604-660) -- primary records of a BGZF
//     BAM in batches; secondary and supplementary records skipped; a record
//     aligned to the reverse strand refused; or the records of a FASTA or
//     FASTQ file, plain or gzip (sniff, FastxReader, fastx_to_record:
//     align.rs:385-563), each taken as an unmapped record; --read-ids
//     (align.rs:572-621); read pairs from two mate files, an interleaved
//     file or a paired BAM (PairSource, align.rs:674-905);
//   * the output records of a read's mapping: build_records
//     (align.rs:1084-1200) with OWNED_TAGS (346-352), int_value (1001-1015),
//     sam_cigar / clipped_span (1017-1052), xa_entry (1054-1069); a read over
//     --max-read-len is written unmapped (process_chunk, 1504-1602); a
//     pair's records: build_pair_records (align.rs:1203-1425) with
//     process_pair_chunk's mate placements (1683-1713);
//   * writing: write_in_order (align.rs:2345-2400) -- chunks in sequence
//     order -- or the coordinate sort (2406-2450): stable on (reference,
//     position, reverse), unmapped last; BGZF blocks with the end marker.
//
// The records are built directly in the BAM layout of the SAM specification
// (section 4.2).  Input tags the CLI does not own are kept byte for byte; the
// owned ones are removed the way its record buffer removes a tag -- the last
// tag moves into the freed slot -- and the new ones appended.  Sequences stay
// in the 4-bit BAM encoding throughout (a reverse hit's read is complemented
// in that encoding).  BGZF blocks are inflated and deflated with zlib on
// several host threads.
#include "../../include/eschalign_b200.h"

#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <unordered_set>
#include <vector>

#include "esg_deflate.cuh"

extern "C" void esg_internal_set_error(esg_status st, const char* msg);

namespace {

esg_status berr(esg_status st, const std::string& msg) {
  esg_internal_set_error(st, msg.c_str());
  return st;
}

uint32_t u32_at(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}
int32_t i32_at(const uint8_t* p) {
  int32_t v;
  memcpy(&v, p, 4);
  return v;
}
uint16_t u16_at(const uint8_t* p) {
  uint16_t v;
  memcpy(&v, p, 2);
  return v;
}
void put32(std::vector<uint8_t>& o, uint32_t v) {
  const size_t n = o.size();
  o.resize(n + 4);
  memcpy(o.data() + n, &v, 4);
}
void put16(std::vector<uint8_t>& o, uint16_t v) {
  const size_t n = o.size();
  o.resize(n + 2);
  memcpy(o.data() + n, &v, 2);
}

uint32_t threads_or(uint32_t t) {
  if (t) return t;
  return std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
}

template <typename F>
void parallel_for(size_t n, uint32_t threads, F&& f) {
  const uint32_t t = (uint32_t)std::min<size_t>(threads, std::max<size_t>(n, 1));
  if (t <= 1) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> th;
  for (uint32_t k = 0; k < t; ++k)
    th.emplace_back([&]() {
      for (size_t i; (i = next.fetch_add(1)) < n;) f(i);
    });
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------- BGZF
constexpr size_t kBgzfMaxIn = 0xff00;  // uncompressed bytes per written block
const uint8_t kBgzfEof[28] = {0x1f, 0x8b, 8, 4, 0, 0, 0, 0, 0, 0xff, 6, 0, 0x42, 0x43,
                              2,    0,    0x1b, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0};

// Inflate BGZF blocks [first, first + n) of `data` (offsets in `starts`)
// into `out`, in order, in parallel.
esg_status inflate_blocks(const std::vector<uint8_t>& data, const std::vector<size_t>& starts,
                          size_t first, size_t n, uint32_t threads, std::vector<uint8_t>& out) {
  std::vector<std::vector<uint8_t>> parts(n);
  std::atomic<int> bad{0};
  parallel_for(n, threads, [&](size_t i) {
    const size_t s = starts[first + i], e = starts[first + i + 1];
    const uint8_t* b = data.data() + s;
    const uint16_t xlen = u16_at(b + 10);
    const size_t cstart = 12 + xlen, clen = (e - s) - cstart - 8;
    const uint32_t isize = u32_at(b + (e - s) - 4);
    if (isize > 65536) {  // a BGZF block holds at most 64 KiB
      bad = 1;
      return;
    }
    parts[i].resize(isize);
    if (!isize) return;
    z_stream z{};
    if (inflateInit2(&z, -15) != Z_OK) {
      bad = 1;
      return;
    }
    z.next_in = const_cast<Bytef*>(b + cstart);
    z.avail_in = (uInt)clen;
    z.next_out = parts[i].data();
    z.avail_out = isize;
    const int rc = inflate(&z, Z_FINISH);
    inflateEnd(&z);
    if (rc != Z_STREAM_END || z.avail_out != 0 ||
        crc32(0L, parts[i].data(), isize) != u32_at(b + (e - s) - 8))
      bad = 1;
  });
  if (bad) return berr(ESG_ERR_BAD_ARGUMENT, "corrupt BGZF block");
  for (auto& p : parts) out.insert(out.end(), p.begin(), p.end());
  return ESG_OK;
}

// A BGZF member: header, the DEFLATE data cdata[0, clen), the CRC32 and
// length of the `n` bytes it holds.
void bgzf_member(const uint8_t* cdata, size_t clen, uint32_t crc, size_t n,
                 std::vector<uint8_t>& out) {
  const uint8_t head[18] = {0x1f, 0x8b, 8, 4, 0, 0, 0, 0, 0, 0xff, 6, 0, 0x42, 0x43, 2, 0, 0, 0};
  out.assign(head, head + 18);
  const uint16_t bsize = (uint16_t)(18 + clen + 8 - 1);
  memcpy(out.data() + 16, &bsize, 2);
  out.insert(out.end(), cdata, cdata + clen);
  put32(out, crc);
  put32(out, (uint32_t)n);
}

// One stored DEFLATE block (BFINAL, BTYPE 00, LEN, NLEN, the bytes) as a
// BGZF member.
void stored_member(const uint8_t* src, size_t n, uint32_t crc, std::vector<uint8_t>& out) {
  std::vector<uint8_t> c = {1, (uint8_t)(n & 0xff), (uint8_t)(n >> 8), (uint8_t)(~n & 0xff),
                            (uint8_t)((~n >> 8) & 0xff)};
  c.insert(c.end(), src, src + n);
  bgzf_member(c.data(), c.size(), crc, n, out);
}

// One BGZF block holding `n` bytes of `src`.
void deflate_block(const uint8_t* src, size_t n, int level, std::vector<uint8_t>& out) {
  z_stream z{};
  deflateInit2(&z, level, Z_DEFLATED, -15, 8, Z_DEFAULT_STRATEGY);
  std::vector<uint8_t> c(deflateBound(&z, (uLong)n) + 32);
  z.next_in = const_cast<Bytef*>(src);
  z.avail_in = (uInt)n;
  z.next_out = c.data();
  z.avail_out = (uInt)c.size();
  deflate(&z, Z_FINISH);
  const size_t clen = c.size() - z.avail_out;
  deflateEnd(&z);
  bgzf_member(c.data(), clen, (uint32_t)crc32(0L, src, (uInt)n), n, out);
}

// ---------------------------------------------------------------- records
// BAM's 4-bit base codes: complement (A<->T, C<->G; anything else N, as the
// reference's letter complement makes it) and to the alphabet's codes 0-4.
const uint8_t kComp4[16] = {15, 8, 4, 15, 2, 15, 15, 15, 1, 15, 15, 15, 15, 15, 15, 15};
const uint8_t kCode4[16] = {4, 0, 1, 4, 2, 4, 4, 4, 3, 4, 4, 4, 4, 4, 4, 4};

struct InRec {  // one input record, `rec` pointing past its block_size
  const uint8_t* rec;
  uint32_t size;
  uint32_t name_len;  // l_read_name (with the NUL)
  uint32_t n_cigar, l_seq;
  uint16_t flag;
  uint32_t aux_off;   // offset of the auxiliary data in rec
  uint32_t seq_off;
};

bool parse_rec(const uint8_t* r, uint32_t size, InRec& x) {
  if (size < 32) return false;
  x.rec = r;
  x.size = size;
  x.name_len = r[8];
  x.n_cigar = u16_at(r + 12);
  x.flag = u16_at(r + 14);
  x.l_seq = u32_at(r + 16);
  // in 64 bits: a corrupt l_seq must not wrap the bound below
  const uint64_t seq_off = 32ull + x.name_len + 4ull * x.n_cigar;
  const uint64_t aux_off = seq_off + (x.l_seq + 1ull) / 2 + x.l_seq;
  if (aux_off > size) return false;
  x.seq_off = (uint32_t)seq_off;
  x.aux_off = (uint32_t)aux_off;
  return true;
}

// (offset, length) of each auxiliary field of a record
bool split_aux(const uint8_t* a, uint32_t n, std::vector<std::pair<uint32_t, uint32_t>>& out) {
  out.clear();
  uint32_t i = 0;
  auto size_of = [](uint8_t t) -> int {
    switch (t) {
      case 'A': case 'c': case 'C': return 1;
      case 's': case 'S': return 2;
      case 'i': case 'I': case 'f': return 4;
      default: return -1;
    }
  };
  while (i < n) {
    if ((uint64_t)i + 3 > n) return false;
    const uint8_t t = a[i + 2];
    uint64_t j = i + 3ull;  // 64 bits: a corrupt array length must not wrap
    if (size_of(t) > 0) {
      j += size_of(t);
    } else if (t == 'Z' || t == 'H') {
      while (j < n && a[j]) ++j;
      ++j;
    } else if (t == 'B') {
      if (j + 5 > n || size_of(a[j]) <= 0) return false;
      j += 5 + (uint64_t)u32_at(a + j + 1) * (uint64_t)size_of(a[j]);
    } else {
      return false;
    }
    if (j > n) return false;
    out.push_back({i, (uint32_t)(j - i)});
    i = (uint32_t)j;
  }
  return true;
}

void int_field(std::vector<uint8_t>& o, const char tag[2], int64_t v) {
  o.push_back((uint8_t)tag[0]);
  o.push_back((uint8_t)tag[1]);
  if (v >= 0 && v <= 255) {
    o.push_back('C');
    o.push_back((uint8_t)v);
  } else if (v >= -128 && v <= 127) {
    o.push_back('c');
    o.push_back((uint8_t)(int8_t)v);
  } else if (v >= 0 && v <= 65535) {
    o.push_back('S');
    put16(o, (uint16_t)v);
  } else if (v >= -32768 && v <= 32767) {
    o.push_back('s');
    put16(o, (uint16_t)(int16_t)v);
  } else if (v >= 0 && v <= 0xffffffffll) {
    o.push_back('I');
    put32(o, (uint32_t)v);
  } else {
    o.push_back('i');
    put32(o, (uint32_t)(int32_t)v);
  }
}

void str_field(std::vector<uint8_t>& o, const char tag[2], const char* s, size_t n) {
  o.push_back((uint8_t)tag[0]);
  o.push_back((uint8_t)tag[1]);
  o.push_back('Z');
  o.insert(o.end(), s, s + n);
  o.push_back(0);
}

uint16_t reg2bin(int64_t beg, int64_t end) {
  --end;
  if (beg >> 14 == end >> 14) return (uint16_t)(((1 << 15) - 1) / 7 + (beg >> 14));
  if (beg >> 17 == end >> 17) return (uint16_t)(((1 << 12) - 1) / 7 + (beg >> 17));
  if (beg >> 20 == end >> 20) return (uint16_t)(((1 << 9) - 1) / 7 + (beg >> 20));
  if (beg >> 23 == end >> 23) return (uint16_t)(((1 << 6) - 1) / 7 + (beg >> 23));
  if (beg >> 26 == end >> 26) return (uint16_t)(((1 << 3) - 1) / 7 + (beg >> 26));
  return 0;
}

// A hit's SAM CIGAR words: soft clips around the aligned span
// (sam_cigar_ad / clipped_span, align.rs:1021-1051).  `ad`: 3' adapter bases
// left out of the alignment, the start of a reverse hit's SEQ.
void sam_cigar(const esg_hit& h, const uint32_t* ops, uint32_t read_len, std::vector<uint32_t>& c,
               uint32_t ad = 0) {
  c.clear();
  const esg_alignment& a = h.alignment;
  const uint32_t shift = h.reverse ? ad : 0;
  const uint32_t qs = a.query_start + shift, qe = a.query_end + shift;
  if (qs > 0) c.push_back(qs << 4 | 4u);
  for (uint32_t k = 0; k < a.n_ops; ++k) c.push_back(ops[a.ops_offset + k]);
  if (read_len > qe) c.push_back((read_len - qe) << 4 | 4u);
}

void cigar_text(const std::vector<uint32_t>& c, std::string& s) {
  for (uint32_t w : c) {
    s += std::to_string(w >> 4);
    s += "MIDNSHP=X"[w & 0xfu];
  }
}

// One record in the BAM layout.  seq4: 4-bit codes, one per byte.  The bin
// is the one noodles' writer (the CLI's) gives: the region [pos, pos + span
// - 1], so a record placed at a position with no CIGAR (an unmapped mate at
// its partner's place) takes [pos, pos - 1]'s bin, and none at position 0.
void encode_record(std::vector<uint8_t>& o, int32_t ref, int32_t pos, uint8_t mapq,
                   const std::vector<uint32_t>& cigar, uint16_t flag, const uint8_t* name,
                   uint32_t name_len, const uint8_t* seq4, uint32_t l_seq, const uint8_t* qual,
                   bool have_qual, const std::vector<uint8_t>& aux, int32_t mate_ref = -1,
                   int32_t mate_pos = -1, int32_t tlen = 0) {
  const size_t at = o.size();
  put32(o, 0);  // block_size, set below
  put32(o, (uint32_t)ref);
  put32(o, (uint32_t)pos);
  uint32_t span = 0;
  for (uint32_t w : cigar) {
    const uint32_t op = w & 0xfu;
    if (op == 0 || op == 2 || op == 3 || op == 7 || op == 8) span += w >> 4;
  }
  const uint16_t bin =
      (pos < 0 || (span == 0 && pos == 0)) ? 4680 : reg2bin(pos, (int64_t)pos + span);
  const uint8_t* nm = name_len > 1 ? name : (const uint8_t*)"*";
  const uint32_t nl = name_len > 1 ? name_len : 2;
  o.push_back((uint8_t)nl);
  o.push_back(mapq);
  put16(o, bin);
  put16(o, (uint16_t)cigar.size());
  put16(o, flag);
  put32(o, l_seq);
  put32(o, (uint32_t)mate_ref);
  put32(o, (uint32_t)mate_pos);
  put32(o, (uint32_t)tlen);
  o.insert(o.end(), nm, nm + nl - 1);
  o.push_back(0);
  for (uint32_t w : cigar) put32(o, w);
  for (uint32_t k = 0; k < l_seq; k += 2)
    o.push_back((uint8_t)(seq4[k] << 4 | (k + 1 < l_seq ? seq4[k + 1] : 0)));
  if (have_qual)
    o.insert(o.end(), qual, qual + l_seq);
  else
    o.insert(o.end(), l_seq, 0xff);
  o.insert(o.end(), aux.begin(), aux.end());
  const uint32_t bs = (uint32_t)(o.size() - at - 4);
  memcpy(o.data() + at, &bs, 4);
}

}  // namespace

// ===================================================================== reader
struct esg_bam_reader {
  FILE* f = nullptr;
  uint32_t threads = 1;
  std::vector<uint8_t> text;
  std::vector<std::string> ref_names;
  std::vector<uint32_t> ref_lens;
  std::vector<uint8_t> buf;  // inflated bytes not yet consumed
  size_t pos = 0;            // consumed prefix of buf
  bool eof = false;
  uint64_t skipped = 0;      // secondary / supplementary records
  // FASTA / FASTQ input (plain or gzip, read through zlib's gz reader)
  int format = 0;            // 0 BAM, 1 FASTA, 2 FASTQ
  gzFile gz = nullptr;
  std::vector<char> lbuf;    // bytes read and not yet split into lines
  size_t lpos = 0, lend = 0;
  bool leof = false;
  uint64_t line_no = 0;
  std::string pending;       // a FASTA header met while ending the previous record
  bool has_pending = false;
  std::string s_header, s_seq, s_qual, s_line;  // next_fastx's scratch
  // paired input: mate 2's file when the mates come in two files
  bool paired = false;
  esg_bam_reader* mate2 = nullptr;
  // --read-ids: the canonical names kept (empty set: no filter)
  std::unordered_set<std::string> wanted;
  bool filter = false;
  uint64_t filtered = 0;
};

struct esg_bam_batch {
  std::vector<uint8_t> bytes;  // the batch's records, each without block_size
  std::vector<InRec> recs;
  std::vector<uint8_t> codes;  // alphabet codes of every read, concatenated
  std::vector<uint64_t> off;
  std::vector<uint32_t> len;
  std::vector<uint32_t> full_len;  // lengths before --max-read-len
};

struct esg_bam_records {
  std::vector<uint8_t> bytes;
  uint32_t n_records = 0;
  // how each read went, the CLI's Outcome (align.rs:1077-1082)
  uint64_t n_unique = 0, n_tied = 0, n_unmapped = 0;
};

// Inflate more blocks into r->buf: up to `want` more blocks, read from the
// file in one go and inflated in parallel.
static esg_status fill(esg_bam_reader* r, size_t want) {
  if (r->eof) return ESG_OK;
  if (r->pos > (1u << 24)) {  // drop the consumed prefix now and then
    r->buf.erase(r->buf.begin(), r->buf.begin() + (long)r->pos);
    r->pos = 0;
  }
  std::vector<uint8_t> data;
  std::vector<size_t> starts{0};
  for (size_t k = 0; k < want; ++k) {
    uint8_t head[18];
    const size_t got = fread(head, 1, 18, r->f);
    if (got == 0) {
      r->eof = true;
      break;
    }
    if (got != 18 || head[0] != 0x1f || head[1] != 0x8b || !(head[3] & 4))
      return berr(ESG_ERR_BAD_ARGUMENT, "not a BGZF file");
    const uint16_t xlen = u16_at(head + 10);
    if (xlen != 6 || head[12] != 'B' || head[13] != 'C')
      return berr(ESG_ERR_BAD_ARGUMENT, "BGZF block without its size field");
    const uint32_t bsize = (uint32_t)u16_at(head + 16) + 1;
    if (bsize < 26) return berr(ESG_ERR_BAD_ARGUMENT, "corrupt BGZF block size");
    const size_t s = data.size();
    data.resize(s + bsize);
    memcpy(data.data() + s, head, 18);
    if (fread(data.data() + s + 18, 1, bsize - 18, r->f) != bsize - 18)
      return berr(ESG_ERR_BAD_ARGUMENT, "truncated BGZF block");
    starts.push_back(data.size());
  }
  if (starts.size() > 1)
    return inflate_blocks(data, starts, 0, starts.size() - 1, r->threads, r->buf);
  return ESG_OK;
}

// At least n unconsumed bytes in r->buf (false at the end of the file).
static esg_status need(esg_bam_reader* r, size_t n, bool* ok) {
  while (r->buf.size() - r->pos < n && !r->eof) {
    const esg_status st = fill(r, (size_t)r->threads * 8);
    if (st != ESG_OK) return st;
  }
  *ok = r->buf.size() - r->pos >= n;
  return ESG_OK;
}

// ------------------------------------------------------------ FASTA / FASTQ
// The CLI's FastxReader (align.rs:436-537), normalise_seq and fastx_to_record
// (align.rs:539-563): multi-line FASTA, four-line FASTQ; a record's name is
// its header up to the first ASCII whitespace; FASTQ qualities are Phred + 33
// (saturating at 0); sequences upper-cased, U read as T, anything outside the
// BAM alphabet as N.  Each record becomes an unmapped BAM record, so the
// encoder treats every input alike.

// Rust's u8::is_ascii_whitespace: space, \t, \n, \x0C, \r.
bool ascii_ws(uint8_t c) { return c == ' ' || c == '\t' || c == '\n' || c == 0x0c || c == '\r'; }

// Next line without its terminator (trailing \n and \r dropped); false at
// the end of the input.
static esg_status next_line(esg_bam_reader* r, std::string& line, bool* got) {
  line.clear();
  *got = false;
  for (;;) {
    if (r->lpos == r->lend) {
      if (r->leof) break;
      const int n = gzread(r->gz, r->lbuf.data(), (unsigned)r->lbuf.size());
      if (n < 0) return berr(ESG_ERR_BAD_ARGUMENT, "reading the input failed (corrupt gzip?)");
      r->lpos = 0;
      r->lend = (size_t)n;
      if (n == 0) {
        r->leof = true;
        break;
      }
    }
    const char* b = r->lbuf.data() + r->lpos;
    const char* nl = (const char*)memchr(b, '\n', r->lend - r->lpos);
    const size_t take = nl ? (size_t)(nl - b) : r->lend - r->lpos;
    line.append(b, take);
    *got = true;
    r->lpos += take;
    if (nl) {
      ++r->lpos;
      break;
    }
  }
  if (*got) {
    ++r->line_no;
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
  }
  return ESG_OK;
}

// Append one FASTX record to `bytes` as an unmapped BAM record (without its
// block_size); false in *got at the end of the input.
static esg_status next_fastx(esg_bam_reader* r, std::vector<uint8_t>& bytes, bool* got) {
  static const std::array<uint8_t, 256> to4 = [] {
    const char* letters = "=ACMGRSVTWYHKDBN";
    std::array<uint8_t, 256> t{};
    t.fill(15);
    for (int k = 0; k < 16; ++k) {
      t[(uint8_t)letters[k]] = (uint8_t)k;
      t[(uint8_t)tolower(letters[k])] = (uint8_t)k;
    }
    t['U'] = t['u'] = 8;  // U as T
    return t;
  }();
  *got = false;
  // the reader's scratch strings keep their capacity from record to record
  std::string& header = r->s_header;
  std::string& seq = r->s_seq;
  std::string& qual = r->s_qual;
  std::string& line = r->s_line;
  header.clear();
  seq.clear();
  qual.clear();
  bool have = false;
  esg_status st;
  const bool fastq = r->format == 2;
  if (!fastq && r->has_pending) {
    header.swap(r->pending);
    r->has_pending = false;
    have = true;
  }
  while (!have) {
    if ((st = next_line(r, line, &have)) != ESG_OK) return st;
    if (!have) return ESG_OK;  // end of input
    if (line.empty()) have = false;
    else header.swap(line);
  }
  const char mark = fastq ? '@' : '>';
  if (header[0] != mark) {
    char m[96];
    snprintf(m, sizeof m, "%s line %llu: expected '%c'", fastq ? "FASTQ" : "FASTA",
             (unsigned long long)r->line_no, mark);
    return berr(ESG_ERR_BAD_ARGUMENT, m);
  }
  size_t ne = 1;
  while (ne < header.size() && !ascii_ws((uint8_t)header[ne])) ++ne;
  const std::string name = header.substr(1, ne - 1);
  if (name.size() > 254) return berr(ESG_ERR_BAD_ARGUMENT, "read name longer than 254 bytes");
  bool qual_given = false;
  if (fastq) {
    if ((st = next_line(r, seq, &have)) != ESG_OK) return st;
    if (!have) return berr(ESG_ERR_BAD_ARGUMENT, "FASTQ truncated after header");
    if ((st = next_line(r, line, &have)) != ESG_OK) return st;
    if (!have || line.empty() || line[0] != '+') {
      char m[64];
      snprintf(m, sizeof m, "FASTQ line %llu: expected '+'", (unsigned long long)r->line_no);
      return berr(ESG_ERR_BAD_ARGUMENT, m);
    }
    if ((st = next_line(r, qual, &have)) != ESG_OK) return st;
    if (!have) return berr(ESG_ERR_BAD_ARGUMENT, "FASTQ truncated before quality");
    if (qual.size() != seq.size()) {
      char m[128];
      snprintf(m, sizeof m, "FASTQ line %llu: %zu quality values for %zu bases",
               (unsigned long long)r->line_no, qual.size(), seq.size());
      return berr(ESG_ERR_BAD_ARGUMENT, m);
    }
    qual_given = true;
  } else {
    for (;;) {
      if ((st = next_line(r, line, &have)) != ESG_OK) return st;
      if (!have) break;
      if (!line.empty() && line[0] == '>') {
        r->pending.swap(line);
        r->has_pending = true;
        break;
      }
      for (char c : line)
        if (!ascii_ws((uint8_t)c)) seq.push_back(c);
    }
  }
  if (seq.size() > 0xffffffffull) return berr(ESG_ERR_BAD_ARGUMENT, "read too long");
  const uint32_t l = (uint32_t)seq.size(), nl = (uint32_t)name.size() + 1;
  put32(bytes, 0xffffffffu);  // reference: none
  put32(bytes, 0xffffffffu);  // position: none
  bytes.push_back((uint8_t)nl);
  bytes.push_back(255);       // mapping quality: missing
  put16(bytes, 4680);
  put16(bytes, 0);            // no CIGAR
  put16(bytes, 0x4);          // unmapped
  put32(bytes, l);
  put32(bytes, 0xffffffffu);
  put32(bytes, 0xffffffffu);
  put32(bytes, 0);
  bytes.insert(bytes.end(), name.begin(), name.end());
  bytes.push_back(0);
  const size_t at = bytes.size();
  bytes.resize(at + (l + 1) / 2 + l);
  uint8_t* d = bytes.data() + at;
  const uint8_t* sq = (const uint8_t*)seq.data();
  for (uint32_t k = 0; k < l; k += 2) *d++ = (uint8_t)(to4[sq[k]] << 4 | (k + 1 < l ? to4[sq[k + 1]] : 0));
  if (qual_given) {
    const uint8_t* qq = (const uint8_t*)qual.data();
    for (uint32_t k = 0; k < l; ++k) d[k] = qq[k] >= 33 ? (uint8_t)(qq[k] - 33) : 0;
  } else {
    memset(d, 0xff, l);
  }
  *got = true;
  return ESG_OK;
}

// The next primary input record, appended to `bytes` without its
// block_size: a BAM's next record that is neither secondary nor
// supplementary (one aligned to the reverse strand is refused), or the next
// FASTX record.  false in *got at the end of the input.
static esg_status next_record(esg_bam_reader* r, std::vector<uint8_t>& bytes, bool* got) {
  *got = false;
  if (r->format != 0) return next_fastx(r, bytes, got);
  for (;;) {
    bool ok = false;
    esg_status st = need(r, 4, &ok);
    if (st != ESG_OK) return st;
    if (!ok) return ESG_OK;
    const uint32_t bs = u32_at(r->buf.data() + r->pos);
    if ((st = need(r, 4 + (size_t)bs, &ok)) != ESG_OK) return st;
    if (!ok) return berr(ESG_ERR_BAD_ARGUMENT, "truncated BAM record");
    const uint8_t* rec = r->buf.data() + r->pos + 4;
    InRec x{};
    if (!parse_rec(rec, bs, x)) return berr(ESG_ERR_BAD_ARGUMENT, "malformed BAM record");
    r->pos += 4 + bs;
    if (x.flag & (0x100 | 0x800)) {  // secondary, supplementary
      ++r->skipped;
      continue;
    }
    if (!(x.flag & 0x4) && (x.flag & 0x10))
      return berr(ESG_ERR_BAD_ARGUMENT,
                  "input record aligned to the reverse strand: unaligned reads (or forward-"
                  "strand alignments, whose SEQ is the read as sequenced) are taken");
    bytes.insert(bytes.end(), rec, rec + bs);
    *got = true;
    return ESG_OK;
  }
}

// A record's name (without its NUL).
static std::string rec_name(const std::vector<uint8_t>& rec) {
  const uint32_t l = rec[8];
  return l > 1 ? std::string((const char*)rec.data() + 32, l - 1) : std::string();
}

// mate_stem (align.rs:700-706): the name without a trailing /1 or /2.
static std::string mate_stem(const std::string& n) {
  if (n.size() >= 2 && n[n.size() - 2] == '/' && (n.back() == '1' || n.back() == '2'))
    return n.substr(0, n.size() - 2);
  return n;
}

// The record with its name replaced.
static void rename_rec(std::vector<uint8_t>& rec, const std::string& name) {
  const uint32_t l = rec[8];
  std::vector<uint8_t> o(rec.begin(), rec.begin() + 32);
  o[8] = (uint8_t)(name.size() + 1);
  o.insert(o.end(), name.begin(), name.end());
  o.push_back(0);
  o.insert(o.end(), rec.begin() + 32 + l, rec.end());
  rec.swap(o);
}

// PairSource::next_pair (align.rs:759-870): the next pair as mate 1, mate 2
// records, both named by the pair's stem (process_pair_chunk,
// align.rs:1631-1639); an orphan mate or a name mismatch is an error
// naming the read.
static esg_status next_pair(esg_bam_reader* r, std::vector<uint8_t>& a, std::vector<uint8_t>& b,
                            bool* got) {
  a.clear();
  b.clear();
  *got = false;
  bool ga = false, gb = false;
  esg_status st;
  if ((st = next_record(r, a, &ga)) != ESG_OK) return st;
  if (r->mate2) {  // two files, record k of each
    if ((st = next_record(r->mate2, b, &gb)) != ESG_OK) return st;
    if (!ga && !gb) return ESG_OK;
    if (ga != gb)
      return berr(ESG_ERR_BAD_ARGUMENT, "read " + rec_name(ga ? a : b) + " has no mate: " +
                                            (ga ? "the mate 2 file" : "the mate 1 file") +
                                            " ends before the other");
    if (mate_stem(rec_name(a)) != mate_stem(rec_name(b)))
      return berr(ESG_ERR_BAD_ARGUMENT, "mate names differ: " + rec_name(a) + " in the mate 1 "
                                        "file but " + rec_name(b) + " in the mate 2 file");
  } else {
    if (!ga) return ESG_OK;
    if (r->format == 0) {
      const uint16_t fa = u16_at(a.data() + 14);
      if (!(fa & 0x1) || !(fa & 0x40) == !(fa & 0x80))
        return berr(ESG_ERR_BAD_ARGUMENT,
                    "read " + rec_name(a) + ": not a mate (paired input needs 0x1 with exactly "
                    "one of 0x40 / 0x80 on every record)");
    }
    if ((st = next_record(r, b, &gb)) != ESG_OK) return st;
    if (!gb) return berr(ESG_ERR_BAD_ARGUMENT, "read " + rec_name(a) + " has no mate: the "
                                                "input ends after it");
    if (mate_stem(rec_name(a)) != mate_stem(rec_name(b)))
      return berr(ESG_ERR_BAD_ARGUMENT, "read " + rec_name(a) + " has no mate: the next record "
                                        "is " + rec_name(b) + " (mates must be adjacent)");
    if (r->format == 0) {
      const uint16_t fa = u16_at(a.data() + 14), fb = u16_at(b.data() + 14);
      if (!(fb & 0x1) || !(fb & 0x40) == !(fb & 0x80) || !(fb & 0x40) == !(fa & 0x40))
        return berr(ESG_ERR_BAD_ARGUMENT, "read " + mate_stem(rec_name(a)) +
                                              ": the two records are not mate 1 and mate 2");
      if (!(fa & 0x40)) a.swap(b);
    }
  }
  const std::string stem = mate_stem(rec_name(a));
  if (stem.size() + 1 != a[8] || memcmp(a.data() + 32, stem.data(), stem.size()) != 0)
    rename_rec(a, stem);
  if (stem.size() + 1 != b[8] || memcmp(b.data() + 32, stem.data(), stem.size()) != 0)
    rename_rec(b, stem);
  *got = true;
  return ESG_OK;
}

// canonical_read_name (align.rs:572-583): a name that parses as a UUID --
// the forms the uuid crate's parse_str takes (32 hex digits, 8-4-4-4-12,
// {8-4-4-4-12}, urn:uuid:8-4-4-4-12; uuid_util.rs:10-30) -- as its dashed
// lower-case string, any other name as it is.
static std::string canonical_read_name(const std::string& n) {
  auto hex = [](char c) { return isxdigit((unsigned char)c) != 0; };
  auto hyphenated = [&](const std::string& t, std::string& h) {
    if (t.size() != 36) return false;
    for (size_t i = 0; i < 36; ++i) {
      if (i == 8 || i == 13 || i == 18 || i == 23) {
        if (t[i] != '-') return false;
      } else if (!hex(t[i])) {
        return false;
      } else {
        h.push_back(t[i]);
      }
    }
    return true;
  };
  std::string h;
  bool ok = false;
  if (n.size() == 32 && std::all_of(n.begin(), n.end(), hex)) {
    h = n;
    ok = true;
  } else if (n.size() == 36) {
    ok = hyphenated(n, h);
  } else if (n.size() == 38 && n.front() == '{' && n.back() == '}') {
    ok = hyphenated(n.substr(1, 36), h);
  } else if (n.size() == 45 && n.compare(0, 9, "urn:uuid:") == 0) {
    ok = hyphenated(n.substr(9), h);
  }
  if (!ok) return n;
  for (char& c : h) c = (char)tolower((unsigned char)c);
  return h.substr(0, 8) + "-" + h.substr(8, 4) + "-" + h.substr(12, 4) + "-" + h.substr(16, 4) +
         "-" + h.substr(20, 12);
}

// Whether --read-ids keeps a read of this name ("*" in a BAM: no name, not
// kept), counting the reads it drops.
static bool kept(esg_bam_reader* r, const std::string& name, bool bam, uint64_t n) {
  if (!r->filter) return true;
  if (!(bam && name == "*") && r->wanted.count(canonical_read_name(name))) return true;
  r->filtered += n;
  return false;
}

// Index a batch's records (bytes complete) and take their reads as
// alphabet codes; a read over max_read_len (0: no limit) gets length 0.
static void finish_batch(esg_bam_batch* b, const std::vector<uint64_t>& rec_off,
                         uint32_t max_read_len) {
  uint64_t total = 0;
  for (size_t k = 0; k < b->recs.size(); ++k) {
    const uint64_t end = k + 1 < rec_off.size() ? rec_off[k + 1] : b->bytes.size();
    InRec& x = b->recs[k];
    parse_rec(b->bytes.data() + rec_off[k], (uint32_t)(end - rec_off[k]), x);
    const bool over = max_read_len && x.l_seq > max_read_len;
    b->full_len.push_back(x.l_seq);
    b->len.push_back(over ? 0u : x.l_seq);
    b->off.push_back(total);
    total += b->len.back();
  }
  b->codes.resize(total);
  for (size_t k = 0; k < b->recs.size(); ++k) {
    const InRec& x = b->recs[k];
    const uint8_t* s = x.rec + x.seq_off;
    uint8_t* d = b->codes.data() + b->off[k];
    for (uint32_t i = 0; i < b->len[k]; ++i) d[i] = kCode4[(s[i / 2] >> ((i & 1) ? 0 : 4)) & 0xf];
  }
}

extern "C" {

esg_status esg_bam_open(const char* path, uint32_t threads, esg_bam_reader** out) {
  if (!path || !out) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  auto* r = new esg_bam_reader();
  r->threads = threads_or(threads);
  r->f = fopen(path, "rb");
  if (!r->f) {
    delete r;
    return berr(ESG_ERR_BAD_ARGUMENT, std::string("cannot open ") + path);
  }
  {
    // sniff (align.rs:385-414): BGZF whose payload starts with BAM\1, or a
    // FASTA / FASTQ, plain or gzip, by its first non-blank character
    uint8_t magic[2] = {0, 0};
    const bool gzip = fread(magic, 1, 2, r->f) == 2 && magic[0] == 0x1f && magic[1] == 0x8b;
    rewind(r->f);
    gzFile g = gzopen(path, "rb");
    if (!g) {
      esg_bam_close(r);
      return berr(ESG_ERR_BAD_ARGUMENT, std::string("cannot open ") + path);
    }
    std::vector<char> head(1 << 16);
    const int n = gzread(g, head.data(), (unsigned)head.size());
    gzclose(g);
    if (n >= 4 && memcmp(head.data(), "BAM\1", 4) == 0) {
      if (!gzip) {
        esg_bam_close(r);
        return berr(ESG_ERR_BAD_ARGUMENT, std::string(path) + ": uncompressed BAM is not supported");
      }
    } else {
      int k = 0;
      while (k < n && ascii_ws((uint8_t)head[k])) ++k;
      if (k == n || (head[k] != '>' && head[k] != '@')) {
        esg_bam_close(r);
        return berr(ESG_ERR_BAD_ARGUMENT,
                    std::string(path) + ": not a BAM, FASTA or FASTQ file (plain or gzip)");
      }
      r->format = head[k] == '>' ? 1 : 2;
      fclose(r->f);
      r->f = nullptr;
      r->gz = gzopen(path, "rb");
      if (!r->gz) {
        esg_bam_close(r);
        return berr(ESG_ERR_BAD_ARGUMENT, std::string("cannot open ") + path);
      }
      gzbuffer(r->gz, 1u << 20);
      r->lbuf.resize(1u << 20);
      *out = r;
      return ESG_OK;
    }
  }
  bool ok = false;
  esg_status st = need(r, 8, &ok);
  auto fail = [&](esg_status s, const char* m) {
    esg_bam_close(r);
    return st != ESG_OK ? st : berr(s, m);
  };
  if (st != ESG_OK || !ok || memcmp(r->buf.data(), "BAM\1", 4) != 0)
    return fail(ESG_ERR_BAD_ARGUMENT, "not a BAM file");
  const uint32_t lt = u32_at(r->buf.data() + 4);
  if ((st = need(r, 12 + (size_t)lt, &ok)) != ESG_OK || !ok)
    return fail(ESG_ERR_BAD_ARGUMENT, "truncated BAM header");
  r->text.assign(r->buf.begin() + 8, r->buf.begin() + 8 + lt);
  r->pos = 8 + lt;
  const uint32_t n_ref = u32_at(r->buf.data() + r->pos);
  r->pos += 4;
  for (uint32_t k = 0; k < n_ref; ++k) {
    if ((st = need(r, 4, &ok)) != ESG_OK || !ok) return fail(ESG_ERR_BAD_ARGUMENT, "truncated");
    const uint32_t ln = u32_at(r->buf.data() + r->pos);
    if ((st = need(r, 8 + (size_t)ln, &ok)) != ESG_OK || !ok)
      return fail(ESG_ERR_BAD_ARGUMENT, "truncated BAM references");
    const char* nm = (const char*)r->buf.data() + r->pos + 4;
    r->ref_names.emplace_back(nm, ln ? ln - 1 : 0);
    r->ref_lens.push_back(u32_at(r->buf.data() + r->pos + 4 + ln));
    r->pos += 8 + ln;
  }
  *out = r;
  return ESG_OK;
}

const char* esg_bam_header_text(const esg_bam_reader* r, uint64_t* len) {
  if (!r) return nullptr;
  if (len) *len = r->text.size();
  return (const char*)r->text.data();
}

esg_status esg_bam_read_batch(esg_bam_reader* r, uint32_t max_reads, uint32_t max_read_len,
                              esg_bam_batch** out) {
  if (!r || !out || !max_reads) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument or batch of 0");
  if (r->paired) return berr(ESG_ERR_BAD_ARGUMENT, "a paired reader: use esg_bam_read_pair_batch");
  *out = nullptr;
  std::unique_ptr<esg_bam_batch> b(new esg_bam_batch());
  std::vector<uint64_t> rec_off;
  while (b->recs.size() < max_reads) {
    const size_t at = b->bytes.size();
    bool got = false;
    const esg_status st = next_record(r, b->bytes, &got);
    if (st != ESG_OK) return st;
    if (!got) break;
    if (r->filter) {
      const uint32_t l = b->bytes[at + 8];
      const std::string name(l > 1 ? (const char*)b->bytes.data() + at + 32 : "", l > 1 ? l - 1 : 0);
      if (!kept(r, name, r->format == 0, 1)) {
        b->bytes.resize(at);
        continue;
      }
    }
    rec_off.push_back(at);
    b->recs.push_back(InRec{});
  }
  finish_batch(b.get(), rec_off, max_read_len);
  *out = b.release();
  return ESG_OK;
}

esg_status esg_bam_read_pair_batch(esg_bam_reader* r, uint32_t max_pairs, esg_bam_batch** out) {
  if (!r || !out || !max_pairs) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument or batch of 0");
  if (!r->paired) return berr(ESG_ERR_BAD_ARGUMENT, "not a paired reader (esg_bam_open_pairs)");
  *out = nullptr;
  std::unique_ptr<esg_bam_batch> b(new esg_bam_batch());
  std::vector<uint64_t> rec_off;
  std::vector<uint8_t> ra, rb;
  while (b->recs.size() < 2 * (size_t)max_pairs) {
    bool got = false;
    const esg_status st = next_pair(r, ra, rb, &got);
    if (st != ESG_OK) return st;
    if (!got) break;
    if (!kept(r, rec_name(ra), false, 2)) continue;
    rec_off.push_back(b->bytes.size());
    b->bytes.insert(b->bytes.end(), ra.begin(), ra.end());
    rec_off.push_back(b->bytes.size());
    b->bytes.insert(b->bytes.end(), rb.begin(), rb.end());
    b->recs.push_back(InRec{});
    b->recs.push_back(InRec{});
  }
  finish_batch(b.get(), rec_off, 0);
  *out = b.release();
  return ESG_OK;
}

esg_status esg_bam_batch_reads(const esg_bam_batch* b, const uint8_t** codes,
                               const uint64_t** off, const uint32_t** len, uint32_t* n_reads) {
  if (!b || !codes || !off || !len || !n_reads) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *codes = b->codes.data();
  *off = b->off.data();
  *len = b->len.data();
  *n_reads = (uint32_t)b->recs.size();
  return ESG_OK;
}

void esg_bam_batch_free(esg_bam_batch* b) { delete b; }

void esg_bam_close(esg_bam_reader* r) {
  if (!r) return;
  if (r->f) fclose(r->f);
  if (r->gz) gzclose(r->gz);
  esg_bam_close(r->mate2);
  delete r;
}

esg_status esg_bam_set_read_ids(esg_bam_reader* r, const char* path) {
  if (!r || !path) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  // load_read_ids (align.rs:585-601): a name per line, its first word; blank
  // lines and lines starting '#' skipped
  gzFile g = gzopen(path, "rb");
  if (!g) return berr(ESG_ERR_BAD_ARGUMENT, std::string("cannot open ") + path);
  std::string text;
  std::vector<char> chunk(1 << 16);
  for (int n; (n = gzread(g, chunk.data(), (unsigned)chunk.size())) > 0;) text.append(chunk.data(), n);
  gzclose(g);
  std::unordered_set<std::string> ids;
  size_t at = 0;
  while (at <= text.size()) {
    size_t e = text.find('\n', at);
    if (e == std::string::npos) e = text.size();
    size_t a = at, z = e;
    while (a < z && ascii_ws((uint8_t)text[a])) ++a;
    while (z > a && ascii_ws((uint8_t)text[z - 1])) --z;
    if (z > a && text[a] != '#') {
      size_t w = a;
      while (w < z && !ascii_ws((uint8_t)text[w])) ++w;
      ids.insert(canonical_read_name(text.substr(a, w - a)));
    }
    at = e + 1;
  }
  if (ids.empty()) return berr(ESG_ERR_BAD_ARGUMENT, std::string("no read names in ") + path);
  r->wanted.swap(ids);
  r->filter = true;
  return ESG_OK;
}

esg_status esg_bam_reader_counts(const esg_bam_reader* r, uint64_t* not_primary,
                                 uint64_t* filtered) {
  if (!r) return berr(ESG_ERR_BAD_ARGUMENT, "NULL reader");
  if (not_primary) *not_primary = r->skipped + (r->mate2 ? r->mate2->skipped : 0);
  if (filtered) *filtered = r->filtered;
  return ESG_OK;
}

esg_status esg_bam_open_pairs(const char* path1, const char* path2, uint32_t threads,
                              esg_bam_reader** out) {
  if (!path1 || !out) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  esg_bam_reader* r = nullptr;
  esg_status st = esg_bam_open(path1, threads, &r);
  if (st != ESG_OK) return st;
  r->paired = true;
  if (path2) {
    if ((st = esg_bam_open(path2, threads, &r->mate2)) != ESG_OK) {
      esg_bam_close(r);
      return st;
    }
    if (r->format == 0 || r->mate2->format == 0) {
      esg_bam_close(r);
      return berr(ESG_ERR_BAD_ARGUMENT, "mates in two files are FASTA / FASTQ; a paired BAM "
                                        "holds both mates in one file");
    }
  }
  *out = r;
  return ESG_OK;
}

// ===================================================================== records
esg_status esg_bam_encode(const esg_bam_batch* b, const esg_mapping* m,
                          const esg_bam_options* opt, const char* const* ref_names,
                          uint32_t n_refs, uint32_t threads, esg_bam_records** out) {
  if (!b || !m || !opt || !out || (n_refs && !ref_names))
    return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  uint32_t n_maps = 0;
  uint64_t n_hits = 0, n_ops = 0, n_md = 0;
  const esg_read_mapping* maps = esg_mapping_reads(m, &n_maps);
  const esg_hit* hits = esg_mapping_hits(m, &n_hits);
  const uint32_t* ops = esg_mapping_ops(m, &n_ops);
  const char* md = esg_mapping_md(m, &n_md);
  if (n_maps != b->recs.size())
    return berr(ESG_ERR_BAD_ARGUMENT, "the mapping is not of this batch's reads");
  const size_t n = b->recs.size();
  for (size_t k = 0; k < n; ++k)
    for (uint32_t h = 0; h < maps[k].n_hits; ++h)
      if (hits[maps[k].first_hit + h].reference >= n_refs)
        return berr(ESG_ERR_BAD_ARGUMENT, "a hit's reference is past ref_names");
  // a scored read's hits lie inside it (a traced hit always does)
  for (size_t k = 0; k < n; ++k)
    if (b->len[k] == b->full_len[k])
      for (uint32_t h = 0; h < maps[k].n_hits; ++h)
        if (hits[maps[k].first_hit + h].alignment.query_end > b->recs[k].l_seq)
          return berr(ESG_ERR_BAD_ARGUMENT, "a hit runs past the end of its read");
  std::vector<std::vector<uint8_t>> enc(n);
  std::vector<uint32_t> count(n, 0), unmapped(n, 0), unique(n, 0);
  std::atomic<int> bad{0};
  parallel_for((n + 63) / 64, threads_or(threads), [&](size_t chunk) {
    std::vector<std::pair<uint32_t, uint32_t>> fields;
    std::vector<uint32_t> cigar;
    std::vector<uint8_t> aux, seq4;
    for (size_t k = chunk * 64; k < std::min(n, chunk * 64 + 64); ++k) {
      const InRec& x = b->recs[k];
      const esg_read_mapping& rm = maps[k];
      std::vector<uint8_t>& o = enc[k];
      const uint8_t* a = x.rec + x.aux_off;
      if (!split_aux(a, x.size - x.aux_off, fields)) {
        bad = 1;
        return;
      }
      // the owned tags removed, each by moving the last field into its slot
      static const char kOwned[5][2] = {{'N', 'M'}, {'M', 'D'}, {'A', 'S'}, {'X', 'S'}, {'X', 'A'}};
      for (const auto& t : kOwned) {
        for (size_t i = 0; i < fields.size(); ++i) {
          if (a[fields[i].first] == (uint8_t)t[0] && a[fields[i].first + 1] == (uint8_t)t[1]) {
            fields[i] = fields.back();
            fields.pop_back();
            break;
          }
        }
      }
      aux.clear();
      for (const auto& fld : fields) aux.insert(aux.end(), a + fld.first, a + fld.first + fld.second);
      const uint16_t kept = x.flag & (0x200 | 0x400);
      const uint8_t* name = x.rec + 32;
      const uint8_t* s = x.rec + x.seq_off;
      const uint8_t* q = s + (x.l_seq + 1) / 2;
      const bool have_qual = x.l_seq == 0 || q[0] != 0xff;
      seq4.resize(x.l_seq);
      for (uint32_t i = 0; i < x.l_seq; ++i) seq4[i] = (s[i / 2] >> ((i & 1) ? 0 : 4)) & 0xf;
      cigar.clear();
      // a read over max_read_len was not scored: unmapped (process_chunk,
      // align.rs:1504-1602)
      if (!rm.n_hits || b->len[k] != b->full_len[k]) {
        encode_record(o, -1, -1, 0, cigar, kept | 0x4, name, x.name_len, seq4.data(), x.l_seq, q,
                      have_qual, aux);
        count[k] = 1;
        unmapped[k] = 1;
        continue;
      }
      const esg_hit& p = hits[rm.first_hit];
      uint16_t flag = kept;
      std::vector<uint8_t> qual(q, q + x.l_seq);
      if (p.reverse) {
        flag |= 0x10;
        std::reverse(seq4.begin(), seq4.end());
        for (auto& c : seq4) c = kComp4[c];
        std::reverse(qual.begin(), qual.end());
      }
      int_field(aux, "NM", p.nm);
      str_field(aux, "MD", md + p.md_offset, p.md_len);
      int_field(aux, "AS", rm.best_score);
      if (rm.flags & ESG_MAPPING_HAS_SUBOPTIMAL) int_field(aux, "XS", rm.suboptimal);
      if (rm.n_hits > 1) {
        std::string xa;
        for (uint32_t h = 1; h < rm.n_hits; ++h) {
          const esg_hit& e = hits[rm.first_hit + h];
          xa += ref_names[e.reference];
          xa += e.reverse ? ",-" : ",+";
          xa += std::to_string(e.alignment.ref_start + 1);
          xa += ',';
          sam_cigar(e, ops, x.l_seq, cigar);
          cigar_text(cigar, xa);
          xa += ',';
          xa += std::to_string(e.nm);
          xa += ';';
        }
        str_field(aux, "XA", xa.data(), xa.size());
      }
      sam_cigar(p, ops, x.l_seq, cigar);
      encode_record(o, (int32_t)p.reference, (int32_t)p.alignment.ref_start,
                    rm.n_tied == 1 ? 60 : 0, cigar, flag, name, x.name_len, seq4.data(), x.l_seq,
                    qual.data(), have_qual, aux);
      count[k] = 1;
      unique[k] = rm.n_tied == 1;
      if (opt->secondary) {
        // the read group of the input record, if any
        std::vector<uint8_t> rg;
        {
          std::vector<std::pair<uint32_t, uint32_t>> all;
          split_aux(a, x.size - x.aux_off, all);
          for (const auto& fld : all)
            if (a[fld.first] == 'R' && a[fld.first + 1] == 'G') {
              rg.assign(a + fld.first, a + fld.first + fld.second);
              break;
            }
        }
        for (uint32_t h = 1; h < rm.n_hits; ++h) {
          const esg_hit& e = hits[rm.first_hit + h];
          std::vector<uint8_t> d;
          int_field(d, "NM", e.nm);
          str_field(d, "MD", md + e.md_offset, e.md_len);
          int_field(d, "AS", rm.best_score);
          d.insert(d.end(), rg.begin(), rg.end());
          sam_cigar(e, ops, x.l_seq, cigar);
          encode_record(o, (int32_t)e.reference, (int32_t)e.alignment.ref_start, 0, cigar,
                        (uint16_t)(0x100 | kept | (e.reverse ? 0x10 : 0)), name, x.name_len,
                        nullptr, 0, nullptr, true, d);
          ++count[k];
        }
      }
    }
  });
  if (bad) return berr(ESG_ERR_BAD_ARGUMENT, "malformed auxiliary data in an input record");
  auto* r = new esg_bam_records();
  size_t total = 0;
  for (auto& e : enc) total += e.size();
  r->bytes.reserve(total);
  for (size_t k = 0; k < n; ++k) {
    r->bytes.insert(r->bytes.end(), enc[k].begin(), enc[k].end());
    r->n_records += count[k];
    r->n_unmapped += unmapped[k];
    r->n_unique += unique[k];
    r->n_tied += !unmapped[k] && !unique[k];
  }
  *out = r;
  return ESG_OK;
}

esg_status esg_bam_encode_pairs(const esg_bam_batch* b, const esg_mapping* m,
                                const uint32_t* adapter_bases, const esg_bam_options* opt,
                                const char* const* ref_names, uint32_t n_refs, uint32_t threads,
                                esg_bam_records** out) {
  if (!b || !m || !opt || !out || (n_refs && !ref_names))
    return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  uint32_t n_pairs = 0, n_maps = 0;
  uint64_t n_phits = 0, n_hits = 0, n_ops = 0, n_md = 0;
  const esg_pair_mapping* pairs = esg_mapping_pairs(m, &n_pairs);
  const esg_pair_hit* phits = esg_mapping_pair_hits(m, &n_phits);
  const esg_read_mapping* maps = esg_mapping_reads(m, &n_maps);
  const esg_hit* hits = esg_mapping_hits(m, &n_hits);
  const uint32_t* ops = esg_mapping_ops(m, &n_ops);
  const char* md = esg_mapping_md(m, &n_md);
  const size_t n = b->recs.size();
  if (n % 2 || (size_t)n_pairs * 2 != n || n_maps != n)
    return berr(ESG_ERR_BAD_ARGUMENT, "the mapping is not of this batch's pairs");
  // every hit's reference named
  for (uint64_t h = 0; h < n_hits; ++h)
    if (hits[h].reference >= n_refs)
      return berr(ESG_ERR_BAD_ARGUMENT, "a hit's reference is past ref_names");
  for (uint64_t h = 0; h < n_phits; ++h)
    if (phits[h].mates[0].reference >= n_refs || phits[h].mates[1].reference >= n_refs)
      return berr(ESG_ERR_BAD_ARGUMENT, "a hit's reference is past ref_names");
  // a Proper pair is placed by its primary pair hit
  for (uint32_t p = 0; p < n_pairs; ++p)
    if ((pairs[p].flags & ESG_PAIR_PROPER) && pairs[p].n_hits == 0)
      return berr(ESG_ERR_BAD_ARGUMENT, "a proper pair has no pair hit");
  // every mate's hit lies inside the mate, its 3' adapter bases around it
  // (a traced hit always does)
  auto outside = [&](const esg_hit& h, size_t mate) {
    const uint32_t shift = (h.reverse && adapter_bases) ? adapter_bases[mate] : 0u;
    return (uint64_t)h.alignment.query_end + shift > b->recs[mate].l_seq;
  };
  for (uint32_t p = 0; p < n_pairs; ++p) {
    for (uint32_t q = 0; q < 2; ++q) {
      const esg_read_mapping& me = maps[2 * (size_t)p + q];
      for (uint32_t h = 0; h < me.n_hits; ++h)
        if (outside(hits[me.first_hit + h], 2 * (size_t)p + q))
          return berr(ESG_ERR_BAD_ARGUMENT, "a hit runs past the end of its mate");
    }
    if (pairs[p].flags & ESG_PAIR_PROPER)
      for (uint32_t t = 0; t < pairs[p].n_hits; ++t)
        for (uint32_t q = 0; q < 2; ++q)
          if (outside(phits[pairs[p].first_hit + t].mates[q], 2 * (size_t)p + q))
            return berr(ESG_ERR_BAD_ARGUMENT, "a pair hit runs past the end of its mate");
  }
  const size_t np = n / 2;
  std::vector<std::vector<uint8_t>> enc(np);
  std::vector<uint32_t> count(np, 0);
  std::vector<uint8_t> outcome(n, 0);  // per mate: 0 unmapped, 1 unique, 2 tied
  std::atomic<int> bad{0};
  static const char kOwned[7][2] = {{'N', 'M'}, {'M', 'D'}, {'A', 'S'}, {'X', 'S'},
                                    {'X', 'A'}, {'M', 'C'}, {'a', 'd'}};
  parallel_for((np + 31) / 32, threads_or(threads), [&](size_t chunk) {
    struct Place {
      const esg_hit* primary = nullptr;
      std::vector<const esg_hit*> others, partners;
      int32_t score = 0;
      bool has_xs = false;
      int32_t xs = 0;
      bool unique = false;
    };
    struct Mate {
      uint16_t kept = 0, flag = 0;
      int32_t ref = -1, pos = -1, mate_ref = -1, mate_pos = -1, tlen = 0;
      uint8_t mapq = 0;
      std::vector<uint32_t> cigar;
      std::vector<uint8_t> seq4, qual, aux, rg;
      bool have_qual = true;
    };
    std::vector<std::pair<uint32_t, uint32_t>> fields;
    std::vector<uint32_t> cig;
    for (size_t p = chunk * 32; p < std::min(np, chunk * 32 + 32); ++p) {
      const esg_pair_mapping& pm = pairs[p];
      const bool proper = pm.flags & ESG_PAIR_PROPER;
      Place pl[2];
      if (proper) {
        const esg_pair_hit* ph = phits + pm.first_hit;
        for (int k = 0; k < 2; ++k) {
          pl[k].primary = &ph[0].mates[k];
          for (uint32_t t = 1; t < pm.n_hits; ++t) {
            pl[k].others.push_back(&ph[t].mates[k]);
            pl[k].partners.push_back(&ph[t].mates[1 - k]);
          }
          pl[k].score = ph[0].mates[k].alignment.score;
          pl[k].has_xs = pm.flags & (k == 0 ? ESG_PAIR_HAS_XS1 : ESG_PAIR_HAS_XS2);
          pl[k].xs = pm.suboptimal[k];
          pl[k].unique = pm.n_tied == 1;
        }
      } else {
        for (int k = 0; k < 2; ++k) {
          const esg_read_mapping& me = maps[2 * p + k];
          const esg_read_mapping& other = maps[2 * p + 1 - k];
          const esg_hit* partner = other.n_hits ? &hits[other.first_hit] : nullptr;
          pl[k].primary = me.n_hits ? &hits[me.first_hit] : nullptr;
          for (uint32_t t = 1; t < me.n_hits; ++t) {
            pl[k].others.push_back(&hits[me.first_hit + t]);
            pl[k].partners.push_back(partner);
          }
          pl[k].score = (me.flags & ESG_MAPPING_HAS_BEST) ? me.best_score : 0;
          pl[k].has_xs = me.flags & ESG_MAPPING_HAS_SUBOPTIMAL;
          pl[k].xs = me.suboptimal;
          pl[k].unique = me.n_tied == 1;
        }
      }
      Mate mt[2];
      uint32_t full[2], ad[2];
      for (int k = 0; k < 2; ++k) {
        const InRec& x = b->recs[2 * p + k];
        full[k] = x.l_seq;
        ad[k] = adapter_bases ? adapter_bases[2 * p + k] : 0u;
        const uint8_t* a = x.rec + x.aux_off;
        if (!split_aux(a, x.size - x.aux_off, fields)) {
          bad = 1;
          return;
        }
        for (const auto& fl : fields)
          if (a[fl.first] == 'R' && a[fl.first + 1] == 'G') {
            mt[k].rg.assign(a + fl.first, a + fl.first + fl.second);
            break;
          }
        for (const auto& t : kOwned)
          for (size_t i = 0; i < fields.size(); ++i)
            if (a[fields[i].first] == (uint8_t)t[0] && a[fields[i].first + 1] == (uint8_t)t[1]) {
              fields[i] = fields.back();
              fields.pop_back();
              break;
            }
        Mate& q = mt[k];
        for (const auto& fl : fields) q.aux.insert(q.aux.end(), a + fl.first, a + fl.first + fl.second);
        q.kept = x.flag & (0x200 | 0x400);
        q.flag = q.kept | 0x1 | (k == 0 ? 0x40 : 0x80);
        const uint8_t* sq = x.rec + x.seq_off;
        const uint8_t* ql = sq + (x.l_seq + 1) / 2;
        q.have_qual = x.l_seq == 0 || ql[0] != 0xff;
        q.seq4.resize(x.l_seq);
        for (uint32_t i = 0; i < x.l_seq; ++i) q.seq4[i] = (sq[i / 2] >> ((i & 1) ? 0 : 4)) & 0xf;
        q.qual.assign(ql, ql + x.l_seq);
        const esg_hit* h = pl[k].primary;
        if (!h) {
          q.flag |= 0x4;
        } else {
          if (h->reverse) {
            q.flag |= 0x10;
            std::reverse(q.seq4.begin(), q.seq4.end());
            for (auto& c : q.seq4) c = kComp4[c];
            std::reverse(q.qual.begin(), q.qual.end());
          }
          q.ref = (int32_t)h->reference;
          q.pos = (int32_t)h->alignment.ref_start;
          q.mapq = pl[k].unique ? 60 : 0;
          sam_cigar(*h, ops, full[k], q.cigar, ad[k]);
          int_field(q.aux, "NM", h->nm);
          str_field(q.aux, "MD", md + h->md_offset, h->md_len);
          int_field(q.aux, "AS", pl[k].score);
          if (pl[k].has_xs) int_field(q.aux, "XS", pl[k].xs);
          if (!pl[k].others.empty()) {
            std::string xa;
            for (const esg_hit* e : pl[k].others) {
              xa += ref_names[e->reference];
              xa += e->reverse ? ",-" : ",+";
              xa += std::to_string(e->alignment.ref_start + 1);
              xa += ',';
              sam_cigar(*e, ops, full[k], cig, ad[k]);
              cigar_text(cig, xa);
              xa += ',';
              xa += std::to_string(e->nm);
              xa += ';';
            }
            str_field(q.aux, "XA", xa.data(), xa.size());
          }
        }
        if (adapter_bases) int_field(q.aux, "ad", ad[k]);
      }
      // template_length (align.rs:1225-1236)
      auto tlen_of = [](const esg_hit& h, const esg_hit& o, bool first) {
        const uint32_t e = std::max(h.alignment.ref_end, o.alignment.ref_end);
        const uint32_t s0 = std::min(h.alignment.ref_start, o.alignment.ref_start);
        const int64_t len = std::min<int64_t>((int64_t)e - s0, INT32_MAX);
        const bool left = h.alignment.ref_start < o.alignment.ref_start ||
                          (h.alignment.ref_start == o.alignment.ref_start && first);
        return (int32_t)(left ? len : -len);
      };
      for (int k = 0; k < 2; ++k) {
        Mate& q = mt[k];
        const esg_hit* h = pl[k].primary;
        const esg_hit* oh = pl[1 - k].primary;
        if (h && oh) {
          if (oh->reverse) q.flag |= 0x20;
          if (proper) q.flag |= 0x2;
          q.mate_ref = (int32_t)oh->reference;
          q.mate_pos = (int32_t)oh->alignment.ref_start;
          std::string mc;
          sam_cigar(*oh, ops, full[1 - k], cig, ad[1 - k]);
          cigar_text(cig, mc);
          str_field(q.aux, "MC", mc.data(), mc.size());
          if (h->reference == oh->reference) q.tlen = tlen_of(*h, *oh, k == 0);
        } else if (h) {
          q.flag |= 0x8;
          q.mate_ref = (int32_t)h->reference;
          q.mate_pos = (int32_t)h->alignment.ref_start;
        } else if (oh) {
          // an unmapped mate sits at its partner's place, as samtools writes it
          if (oh->reverse) q.flag |= 0x20;
          q.ref = q.mate_ref = (int32_t)oh->reference;
          q.pos = q.mate_pos = (int32_t)oh->alignment.ref_start;
        } else {
          q.flag |= 0x8;
        }
      }
      std::vector<uint8_t>& o = enc[p];
      for (int k = 0; k < 2; ++k)
        outcome[2 * p + k] = !pl[k].primary ? 0 : (pl[k].unique ? 1 : 2);
      for (int k = 0; k < 2; ++k) {
        const InRec& x = b->recs[2 * p + k];
        const Mate& q = mt[k];
        encode_record(o, q.ref, q.pos, q.mapq, q.cigar, q.flag, x.rec + 32, x.name_len,
                      q.seq4.data(), x.l_seq, q.qual.data(), q.have_qual, q.aux, q.mate_ref,
                      q.mate_pos, q.tlen);
      }
      count[p] = 2;
      if (opt->secondary) {
        const size_t nt = std::max(pl[0].others.size(), pl[1].others.size());
        for (size_t t = 0; t < nt; ++t)
          for (int k = 0; k < 2; ++k) {
            if (t >= pl[k].others.size()) continue;
            const esg_hit& h = *pl[k].others[t];
            const esg_hit* ph = pl[k].partners[t];
            uint16_t f = 0x100 | 0x1 | (k == 0 ? 0x40 : 0x80) | mt[k].kept;
            if (h.reverse) f |= 0x10;
            std::vector<uint8_t> d;
            int_field(d, "NM", h.nm);
            str_field(d, "MD", md + h.md_offset, h.md_len);
            int_field(d, "AS", h.alignment.score);
            d.insert(d.end(), mt[k].rg.begin(), mt[k].rg.end());
            int32_t mref = (int32_t)h.reference, mpos = (int32_t)h.alignment.ref_start, tl = 0;
            if (ph) {
              if (ph->reverse) f |= 0x20;
              mref = (int32_t)ph->reference;
              mpos = (int32_t)ph->alignment.ref_start;
              if (proper) {
                f |= 0x2;
                if (ph->reference == h.reference) tl = tlen_of(h, *ph, k == 0);
              }
            } else {
              f |= 0x8;
            }
            sam_cigar(h, ops, full[k], cig, ad[k]);
            const InRec& x = b->recs[2 * p + k];
            encode_record(o, (int32_t)h.reference, (int32_t)h.alignment.ref_start, 0, cig, f,
                          x.rec + 32, x.name_len, nullptr, 0, nullptr, true, d, mref, mpos, tl);
            ++count[p];
          }
      }
    }
  });
  if (bad) return berr(ESG_ERR_BAD_ARGUMENT, "malformed auxiliary data in an input record");
  auto* r = new esg_bam_records();
  size_t total = 0;
  for (auto& e : enc) total += e.size();
  r->bytes.reserve(total);
  for (size_t p = 0; p < np; ++p) {
    r->bytes.insert(r->bytes.end(), enc[p].begin(), enc[p].end());
    r->n_records += count[p];
  }
  for (uint8_t oc : outcome) {
    r->n_unmapped += oc == 0;
    r->n_unique += oc == 1;
    r->n_tied += oc == 2;
  }
  *out = r;
  return ESG_OK;
}

const uint8_t* esg_bam_records_bytes(const esg_bam_records* r, uint64_t* n_bytes,
                                     uint32_t* n_records) {
  if (!r) return nullptr;
  if (n_bytes) *n_bytes = r->bytes.size();
  if (n_records) *n_records = r->n_records;
  return r->bytes.data();
}

esg_status esg_bam_records_outcomes(const esg_bam_records* r, uint64_t* unique, uint64_t* tied,
                                    uint64_t* unmapped) {
  if (!r) return berr(ESG_ERR_BAD_ARGUMENT, "NULL records");
  if (unique) *unique = r->n_unique;
  if (tied) *tied = r->n_tied;
  if (unmapped) *unmapped = r->n_unmapped;
  return ESG_OK;
}

void esg_bam_records_free(esg_bam_records* r) { delete r; }

}  // extern "C"

// ===================================================================== writer
// Blocks deflated on a device (esg_deflate.cuh): one job in flight.  A job
// is the whole blocks of one drain: uploaded, compressed by k_bgzf_deflate
// on a stream of the highest priority, and copied back; the next drain (or
// the close) writes them, so the device's work overlaps the host's next
// chunk.  Each block's CRC32 is computed on the host while the device
// compresses.
struct DeviceDeflate {
  int device = -1;
  cudaStream_t stream = nullptr;
  uint8_t* d_in = nullptr;
  uint32_t* d_tok = nullptr;
  uint32_t* d_out = nullptr;
  uint32_t* d_len = nullptr;
  uint8_t* h_out = nullptr;  // pinned
  uint32_t* h_len = nullptr;  // pinned
  size_t cap = 0;             // blocks the buffers hold
  size_t nb = 0;              // blocks of the job in flight (0: none)
  size_t bytes = 0;           // its input bytes
  std::vector<uint32_t> crc;
  uint64_t blocks = 0, stored = 0;  // blocks written, of them stored
};

struct esg_bam_writer {
  FILE* f = nullptr;
  uint32_t threads = 1;
  int level = 6;
  bool sort = false;
  std::vector<uint8_t> pending;  // uncompressed bytes not yet in a block
  std::map<uint64_t, std::vector<uint8_t>> waiting;  // chunks ahead of `next`
  uint64_t next = 0;
  std::vector<std::vector<uint8_t>> buckets;  // coordinate sort: per reference, + unmapped
  bool failed = false;
  std::unique_ptr<DeviceDeflate> dev;
};

static esg_status cuda_fail(esg_bam_writer* w, cudaError_t e, const char* what) {
  w->failed = true;
  return berr(ESG_ERR_DRIVER, std::string("device deflate: ") + what + ": " +
                                  cudaGetErrorString(e));
}

static void device_free(DeviceDeflate& D) {
  if (D.device < 0) return;
  cudaSetDevice(D.device);
  if (D.stream) cudaStreamSynchronize(D.stream);
  cudaFree(D.d_in);
  cudaFree(D.d_tok);
  cudaFree(D.d_out);
  cudaFree(D.d_len);
  cudaFreeHost(D.h_out);
  cudaFreeHost(D.h_len);
  if (D.stream) cudaStreamDestroy(D.stream);
  D = DeviceDeflate{};
}

// Write the blocks of the job in flight.
static esg_status device_finish(esg_bam_writer* w) {
  DeviceDeflate& D = *w->dev;
  if (!D.nb) return ESG_OK;
  cudaError_t e = cudaSetDevice(D.device);
  if (e == cudaSuccess) e = cudaStreamSynchronize(D.stream);
  if (e != cudaSuccess) return cuda_fail(w, e, "compressing");
  namespace dz = esg_deflate;
  std::vector<uint8_t> member, raw;
  for (size_t i = 0; i < D.nb; ++i) {
    const size_t n = std::min<size_t>(kBgzfMaxIn, D.bytes - i * kBgzfMaxIn);
    const uint32_t clen = D.h_len[i];
    if (clen == dz::kStored) {  // incompressible: the input, from the device
      raw.resize(n);
      e = cudaMemcpyAsync(raw.data(), D.d_in + i * kBgzfMaxIn, n, cudaMemcpyDeviceToHost,
                          D.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(D.stream);
      if (e != cudaSuccess) return cuda_fail(w, e, "reading a stored block back");
      stored_member(raw.data(), n, D.crc[i], member);
      ++D.stored;
    } else {
      if (clen > n + 5) {
        w->failed = true;
        return berr(ESG_ERR_DRIVER, "device deflate: block length out of range");
      }
      bgzf_member(D.h_out + i * dz::kSlotBytes, clen, D.crc[i], n, member);
    }
    if (fwrite(member.data(), 1, member.size(), w->f) != member.size()) {
      w->failed = true;
      return berr(ESG_ERR_DRIVER, "writing the BAM file failed");
    }
  }
  D.blocks += D.nb;
  D.nb = 0;
  return ESG_OK;
}

// Start a job on w->pending[0, whole).
static esg_status device_start(esg_bam_writer* w, size_t whole) {
  DeviceDeflate& D = *w->dev;
  namespace dz = esg_deflate;
  const size_t nb = (whole + kBgzfMaxIn - 1) / kBgzfMaxIn;
  cudaError_t e = cudaSetDevice(D.device);
  if (e != cudaSuccess) return cuda_fail(w, e, "selecting the device");
  if (!D.stream) {
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    e = cudaStreamCreateWithPriority(&D.stream, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(dz::k_bgzf_deflate, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(dz::BlockState));
    if (e != cudaSuccess) return cuda_fail(w, e, "creating the stream");
  }
  if (nb > D.cap) {
    cudaFree(D.d_in);
    cudaFree(D.d_tok);
    cudaFree(D.d_out);
    cudaFree(D.d_len);
    cudaFreeHost(D.h_out);
    cudaFreeHost(D.h_len);
    D.d_in = nullptr;
    D.d_tok = D.d_out = D.d_len = D.h_len = nullptr;
    D.h_out = nullptr;
    D.cap = 0;
    const size_t cap = std::max<size_t>(nb, 64);
    e = cudaMalloc(&D.d_in, cap * kBgzfMaxIn);
    if (e == cudaSuccess) e = cudaMalloc(&D.d_tok, cap * dz::kTokensPerBlock * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&D.d_out, cap * dz::kSlotBytes);
    if (e == cudaSuccess) e = cudaMalloc(&D.d_len, cap * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaHostAlloc(&D.h_out, cap * dz::kSlotBytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&D.h_len, cap * sizeof(uint32_t), cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(w, e, "allocating buffers");
    D.cap = cap;
  }
  e = cudaMemcpyAsync(D.d_in, w->pending.data(), whole, cudaMemcpyHostToDevice, D.stream);
  if (e != cudaSuccess) return cuda_fail(w, e, "uploading");
  dz::k_bgzf_deflate<<<(unsigned)nb, dz::kLanes, sizeof(dz::BlockState), D.stream>>>(
      D.d_in, whole, D.d_tok, D.d_out, D.d_len);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(D.h_len, D.d_len, nb * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        D.stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(D.h_out, D.d_out, nb * dz::kSlotBytes, cudaMemcpyDeviceToHost, D.stream);
  if (e != cudaSuccess) return cuda_fail(w, e, "launching");
  D.crc.assign(nb, 0);
  parallel_for(nb, w->threads, [&](size_t i) {
    const size_t n = std::min<size_t>(kBgzfMaxIn, whole - i * kBgzfMaxIn);
    D.crc[i] = (uint32_t)crc32(0L, w->pending.data() + i * kBgzfMaxIn, (uInt)n);
  });
  D.nb = nb;
  D.bytes = whole;
  return ESG_OK;
}

// Compress every whole block of w->pending (all of it with `flush`) and
// write them in order.
static esg_status drain(esg_bam_writer* w, bool flush) {
  const size_t whole = flush ? w->pending.size() : w->pending.size() / kBgzfMaxIn * kBgzfMaxIn;
  if (w->dev) {
    esg_status st = device_finish(w);
    if (st == ESG_OK && whole) {
      st = device_start(w, whole);
      if (st == ESG_OK) w->pending.erase(w->pending.begin(), w->pending.begin() + (long)whole);
    }
    if (st == ESG_OK && flush) st = device_finish(w);
    return st;
  }
  if (!whole) return ESG_OK;
  const size_t nb = (whole + kBgzfMaxIn - 1) / kBgzfMaxIn;
  std::vector<std::vector<uint8_t>> blocks(nb);
  parallel_for(nb, w->threads, [&](size_t i) {
    const size_t s = i * kBgzfMaxIn;
    deflate_block(w->pending.data() + s, std::min(kBgzfMaxIn, whole - s), w->level, blocks[i]);
  });
  for (auto& bl : blocks)
    if (fwrite(bl.data(), 1, bl.size(), w->f) != bl.size()) {
      w->failed = true;
      return berr(ESG_ERR_DRIVER, "writing the BAM file failed");
    }
  w->pending.erase(w->pending.begin(), w->pending.begin() + (long)whole);
  return ESG_OK;
}

static void put_records(esg_bam_writer* w, const uint8_t* p, size_t n) {
  if (!w->sort) {
    w->pending.insert(w->pending.end(), p, p + n);
    return;
  }
  for (size_t at = 0; at + 4 <= n;) {
    const uint32_t bs = u32_at(p + at);
    const int32_t tid = i32_at(p + at + 4);
    const size_t b = (tid >= 0 && (size_t)tid < w->buckets.size() - 1) ? (size_t)tid
                                                                          : w->buckets.size() - 1;
    w->buckets[b].insert(w->buckets[b].end(), p + at, p + at + 4 + bs);
    at += 4 + bs;
  }
}

extern "C" {

esg_status esg_bam_writer_open(const char* path, const char* header_text,
                               const char* const* ref_names, const uint32_t* ref_lens,
                               uint32_t n_refs, int32_t sort_coordinate, uint32_t threads,
                               esg_bam_writer** out) {
  if (!path || !out || (n_refs && (!ref_names || !ref_lens)))
    return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  *out = nullptr;
  auto* w = new esg_bam_writer();
  w->threads = threads_or(threads);
  w->sort = sort_coordinate != 0;
  w->buckets.resize((size_t)n_refs + 1);
  w->f = fopen(path, "wb");
  if (!w->f) {
    delete w;
    return berr(ESG_ERR_BAD_ARGUMENT, std::string("cannot create ") + path);
  }
  const size_t lt = header_text ? strlen(header_text) : 0;
  std::vector<uint8_t>& h = w->pending;
  h.insert(h.end(), {'B', 'A', 'M', 1});
  put32(h, (uint32_t)lt);
  h.insert(h.end(), header_text, header_text + lt);
  put32(h, n_refs);
  for (uint32_t k = 0; k < n_refs; ++k) {
    const size_t ln = strlen(ref_names[k]) + 1;
    put32(h, (uint32_t)ln);
    h.insert(h.end(), ref_names[k], ref_names[k] + ln);
    put32(h, ref_lens[k]);
  }
  *out = w;
  return ESG_OK;
}

esg_status esg_bam_writer_push(esg_bam_writer* w, uint64_t seq, const esg_bam_records* r) {
  if (!w || !r) return berr(ESG_ERR_BAD_ARGUMENT, "NULL argument");
  if (w->failed) return berr(ESG_ERR_DRIVER, "the writer failed earlier");
  if (seq < w->next || w->waiting.count(seq))
    return berr(ESG_ERR_BAD_ARGUMENT, "chunk sequence number already written");
  w->waiting[seq] = r->bytes;
  for (auto it = w->waiting.find(w->next); it != w->waiting.end(); it = w->waiting.find(w->next)) {
    put_records(w, it->second.data(), it->second.size());
    w->waiting.erase(it);
    ++w->next;
  }
  return drain(w, false);
}

esg_status esg_bam_writer_close(esg_bam_writer* w) {
  if (!w) return berr(ESG_ERR_BAD_ARGUMENT, "NULL writer");
  esg_status st = ESG_OK;
  if (!w->waiting.empty()) st = berr(ESG_ERR_BAD_ARGUMENT, "chunks missing before the last pushed");
  if (st == ESG_OK && w->sort) {
    // per reference, stable on (position, reverse): records are pushed in
    // input order, so ties keep it
    for (size_t bkt = 0; bkt < w->buckets.size() && st == ESG_OK; ++bkt) {
      std::vector<uint8_t>& v = w->buckets[bkt];
      std::vector<std::pair<uint64_t, size_t>> keyed;
      for (size_t at = 0; at + 4 <= v.size(); at += 4 + u32_at(v.data() + at)) {
        const bool unmapped = bkt == w->buckets.size() - 1;
        const uint64_t pos = unmapped ? 0 : (uint64_t)(uint32_t)i32_at(v.data() + at + 8);
        const uint64_t rev = (u16_at(v.data() + at + 18) & 0x10) ? 1 : 0;
        keyed.push_back({pos << 1 | rev, at});
      }
      std::stable_sort(keyed.begin(), keyed.end(),
                       [](const std::pair<uint64_t, size_t>& a,
                          const std::pair<uint64_t, size_t>& b) { return a.first < b.first; });
      for (const auto& kv : keyed) {
        const uint32_t bs = u32_at(v.data() + kv.second);
        w->pending.insert(w->pending.end(), v.data() + kv.second, v.data() + kv.second + 4 + bs);
      }
      std::vector<uint8_t>().swap(v);
      st = drain(w, false);
    }
  }
  if (st == ESG_OK) st = drain(w, true);
  if (st == ESG_OK && fwrite(kBgzfEof, 1, sizeof kBgzfEof, w->f) != sizeof kBgzfEof)
    st = berr(ESG_ERR_DRIVER, "writing the BAM file failed");
  if (fclose(w->f) != 0 && st == ESG_OK) st = berr(ESG_ERR_DRIVER, "closing the BAM file failed");
  if (w->dev) device_free(*w->dev);
  delete w;
  return st;
}

esg_status esg_bam_writer_use_device(esg_bam_writer* w, int32_t device) {
  if (!w) return berr(ESG_ERR_BAD_ARGUMENT, "NULL writer");
  if (w->failed) return berr(ESG_ERR_DRIVER, "the writer failed earlier");
  if (device < 0) {  // back to the host threads
    if (w->dev) {
      const esg_status st = device_finish(w);
      device_free(*w->dev);
      w->dev.reset();
      return st;
    }
    return ESG_OK;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device >= count)
    return berr(ESG_ERR_BAD_ARGUMENT, "esg_bam_writer_use_device: no such device");
  if (w->dev && w->dev->device != device) {
    const esg_status st = device_finish(w);
    if (st != ESG_OK) return st;
    device_free(*w->dev);
    w->dev.reset();
  }
  if (!w->dev) {
    w->dev.reset(new DeviceDeflate);
    w->dev->device = device;
  }
  return ESG_OK;
}

esg_status esg_bam_writer_blocks(const esg_bam_writer* w, uint64_t* blocks,
                                 uint64_t* stored) {
  if (!w) return berr(ESG_ERR_BAD_ARGUMENT, "NULL writer");
  if (blocks) *blocks = w->dev ? w->dev->blocks : 0;
  if (stored) *stored = w->dev ? w->dev->stored : 0;
  return ESG_OK;
}

// The device deflate's steps run on the host, lane by lane: one block of at
// most 0xff00 bytes into `out` (65536 bytes, 4-byte aligned).  Returns the
// DEFLATE length, 0xffffffff for "store it", 0 on a bad argument.  A check
// of the steps for tests; the writer never calls it.
uint32_t esg_bgzf_deflate_host(const uint8_t* src, uint32_t n, uint8_t* out) {
  namespace dz = esg_deflate;
  if (!src || !out || n == 0 || n > dz::kBlockIn) return 0;
  std::unique_ptr<dz::BlockState> S(new dz::BlockState);
  std::vector<uint32_t> tok(dz::kTokensPerBlock);
  return dz::deflate_block_host(src, n, out, *S, tok.data());
}

// The compressor's code lengths on the host: freq[0, n) (n <= 288) to
// lengths of at most `limit` (1..15) bits.  Returns 0, or -1 on a bad
// argument.  A check of the step for tests.
int32_t esg_bgzf_code_lengths(const uint32_t* freq, uint32_t n, uint32_t limit, uint8_t* len) {
  namespace dz = esg_deflate;
  if (!freq || !len || n < 2 || n > dz::kMaxSyms || limit < 1 || limit > 15) return -1;
  uint64_t m = 0;
  for (uint32_t i = 0; i < n; ++i) m += freq[i] != 0;
  if (m > (1ull << limit)) return -1;  // more symbols than codes of that length
  std::unique_ptr<dz::BlockState> S(new dz::BlockState);
  dz::huffman_lengths(freq, n, limit, len, *S);
  return 0;
}

}  // extern "C"
