/*
 * esg_oracle.h -- CPU restatement of eschalign's panel-scoring path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against (tests/, __graft_entry__.smoke(), and bench.py's
 * cpu_baseline leg and `--impl reference` arm).  Nothing in the product
 * (eschalign_b200/) links, loads or calls it.
 *
 * Parity is pinned: the scalar score is checked against the reference's 192
 * parasail golden scores (tests/golden/align_golden_scores.json, extracted
 * from crates/eschalign/tests/fixtures/align_golden.json by
 * tests/golden/make_golden.py) and the unit known-answers of
 * crates/eschalign/src/scalar.rs:378-430 and mapper.rs:570-589.
 *
 * Two scorers live here:
 *   - eo_score: the scalar Gotoh (crates/eschalign/src/scalar.rs:120-163),
 *     the oracle every other path must equal;
 *   - eo_profile_*: the AVX-512BW inter-sequence kernels of
 *     crates/eschalign/src/simd/avx512.rs (row-major :43-107, transposed
 *     :278-354) with the reference's dispatch (mapper.rs:216-222,
 *     simd/mod.rs:222-227), the timed CPU baseline.
 */
#ifndef ESG_ORACLE_H
#define ESG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Codes of crates/eschalign/src/alphabet.rs:7-16. */
enum { EO_A = 0, EO_C = 1, EO_G = 2, EO_T = 3, EO_WILDCARD = 4, EO_N_CODES = 5 };

/* Same layout as the product's esg_read_result (include/eschalign_b200.h). */
typedef struct eo_result {
    int32_t best;       /* max over the read's candidates                     */
    int32_t suboptimal; /* best score not equal to `best`; INT32_MIN if none  */
    uint32_t n_tied;    /* candidates scoring `best`                           */
    uint32_t flags;     /* EO_RESULT_* */
} eo_result;

#define EO_NO_SCORE INT32_MIN
#define EO_RESULT_EMPTY 1u          /* empty read: no candidates at all         */
#define EO_RESULT_TIES_TRUNCATED 2u /* n_tied exceeds the tie list's capacity  */

/* alphabet.rs:29-50: A/C/G/T(U) either case -> 0..3, every other byte -> 4. */
uint8_t eo_encode_base(uint8_t letter);
void eo_encode(const uint8_t* letters, size_t n, uint8_t* codes);
/* alphabet.rs:58-64: reverse, complement c -> 3-c, the wildcard stays. */
void eo_revcomp_codes(const uint8_t* codes, size_t n, uint8_t* out);

/* scoring.rs:70-100.  0 = valid; 1 match <= 0; 2 mismatch >= match;
 * 3 a gap score > 0; 4 a magnitude above 1000. */
int eo_scoring_validate(int32_t ma, int32_t mi, int32_t o, int32_t e);

/* scalar.rs:120-163: best Gotoh score of query (n codes) vs reference (m). */
int32_t eo_score(const uint8_t* q, size_t n, const uint8_t* r, size_t m,
                 int32_t ma, int32_t mi, int32_t o, int32_t e, int local);

/* simd/mod.rs:222-227 */
int eo_fits_i16(size_t n, size_t max_ref_len, int32_t ma, int32_t mi, int32_t o, int32_t e);

/* mapper.rs:444-472: candidates in order (ref 0 fwd, ref 0 rev, ref 1 fwd, ...);
 * `rev` may be NULL (forward strand only).  Writes the first min(n_tied, cap)
 * tie candidates as (ref << 1) | reverse into `ties`. */
void eo_select(const int32_t* fwd, const int32_t* rev, uint32_t n_refs, uint32_t cap,
               eo_result* out, uint32_t* ties);

/* Every query against every reference with eo_score, out[q * n_refs + r];
 * `threads` <= 0 uses all cores. */
void eo_score_matrix(const uint8_t* codes, const uint64_t* off, const uint32_t* len, uint32_t n_q,
                     const uint8_t* ref_codes, const uint64_t* ref_off, const uint32_t* ref_len,
                     uint32_t n_refs, int32_t ma, int32_t mi, int32_t o, int32_t e, int local,
                     int threads, int32_t* out);

/* ---- AVX-512BW baseline (simd/mod.rs + simd/avx512.rs) ---------------- */
typedef struct eo_profile eo_profile;

/* Profile::from_codes (simd/mod.rs:292-331) at 32 lanes, plus the transposed
 * profile (simd/mod.rs:255-269).  NULL if the CPU lacks AVX-512BW. */
eo_profile* eo_profile_build(const uint8_t* ref_codes, const uint64_t* ref_off,
                             const uint32_t* ref_len, uint32_t n_refs,
                             int32_t ma, int32_t mi, int32_t o, int32_t e);
void eo_profile_free(eo_profile* p);
int eo_cpu_has_avx512bw(void);

/* Aligner::score_all (mapper.rs:242-252): SIMD when fits_i16, row-major
 * below 256 nt and transposed from 256 nt (kernel = 0), or forced
 * (1 row-major, 2 transposed); scalar outside fits_i16. out[n_refs]. */
void eo_profile_score_all(const eo_profile* p, const uint8_t* q, size_t n, int local,
                          int kernel, int32_t* out);

/* The CPU baseline end to end: per read, score the forward strand (and the
 * reverse complement when both_strands), then eo_select.  Reads are handed
 * out to `threads` workers (<= 0: all cores) in chunks of 64 reads
 * (crates/eschalign-cli/src/align.rs:1470-1473).  Returns the thread count
 * used.  `rows`, when not NULL, receives every query's scores: forward rows
 * 0..n-1 then reverse rows n..2n-1. */
int eo_cpu_map_batch(const eo_profile* p, const uint8_t* codes, const uint64_t* off,
                     const uint32_t* len, uint32_t n_reads, int both_strands, int local,
                     int threads, uint32_t cap, eo_result* results, uint32_t* ties,
                     int32_t* rows);

/* Reads per work unit of eo_cpu_map_batch's workers (default 64). */
void eo_cpu_set_chunk(int reads);

/* Same, with the scalar oracle instead of the SIMD kernels (used at test
 * sizes; identical results by construction of the reference). */
int eo_scalar_map_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                        uint32_t n_reads, const uint8_t* ref_codes, const uint64_t* ref_off,
                        const uint32_t* ref_len, uint32_t n_refs, int32_t ma, int32_t mi,
                        int32_t o, int32_t e, int both_strands, int local, int threads,
                        uint32_t cap, eo_result* results, uint32_t* ties, int32_t* rows);

/* ---- paired-end (adapter.rs, mapper/pair.rs) --------------------------- */
/* adapter.rs:68-91 on codes: adapter bases at the 3' end of `read` (0 = none). */
size_t eo_adapter_find(const uint8_t* read, size_t n, const uint8_t* adapter, size_t a,
                       size_t min_overlap);
/* adapter.rs:95-110: out = {ad1, ad2}, the two mates' insert ends reconciled. */
void eo_adapter_detect_pair(const uint8_t* r1, size_t l1, const uint8_t* r2, size_t l2,
                            const uint8_t* a1, size_t al1, const uint8_t* a2, size_t al2,
                            size_t min_overlap, size_t out[2]);
/* align.rs:934-949 (pair_adapters), with the over-length rule. */
void eo_pair_adapters(const uint8_t* r1, size_t l1, const uint8_t* r2, size_t l2,
                      const uint8_t* a1, size_t al1, const uint8_t* a2, size_t al2,
                      size_t min_overlap, size_t max_read_len, size_t out[2]);

/* Same layout as the product's esg_pair_result. */
typedef struct eo_pair_result {
    int32_t best;       /* best summed mate score; INT32_MIN if no candidate   */
    int32_t next;       /* the next tier's sum; INT32_MIN if none               */
    uint32_t n_tied;    /* candidates in the first tier                         */
    uint32_t flags;     /* EO_RESULT_EMPTY: no eligible candidate; TRUNCATED    */
    int32_t xs[2];      /* per mate: best over candidates outside the tier     */
    int32_t primary[2]; /* the first tie's mate scores                          */
} eo_pair_result;

/* pair.rs:195-234 and :297-314.  f0/r0: mate 1 forward / reverse-complement
 * row, f1/r1 mate 2's.  Ties as (ref << 1) | template_reverse. */
void eo_pair_select(const int32_t* f0, const int32_t* r0, const int32_t* f1, const int32_t* r1,
                    uint32_t n_refs, int both_strands, int32_t min_score, uint32_t cap,
                    eo_pair_result* out, uint32_t* ties);
/* The ranking over rows in the CUDA path's layout (forward rows of the
 * 2 n_pairs mates, then their reverse-complement rows); len = mate lengths. */
void eo_pairs_from_rows(const int32_t* rows, const uint32_t* len, uint32_t n_pairs,
                        uint32_t n_refs, int both_strands, int32_t min_score, uint32_t cap,
                        eo_pair_result* results, uint32_t* ties);
/* The reference's CPU path for pairs (the timed baseline): trimming, the
 * four mate rows with the SIMD kernels, the pair ranking and each mate's
 * both-strand selection, OpenMP over pairs.  Returns the thread count. */
int eo_cpu_map_pairs(const eo_profile* p, const uint8_t* codes, const uint64_t* off,
                     const uint32_t* len, uint32_t n_pairs, const uint8_t* a1, size_t al1,
                     const uint8_t* a2, size_t al2, size_t min_overlap, size_t max_read_len,
                     int both_strands, int local, int32_t min_score, int threads, uint32_t cap,
                     eo_pair_result* results, uint32_t* ties, eo_result* mate_results,
                     uint32_t* mate_ties, uint32_t* adapters);
/* Pairs end to end with the scalar oracle; mates 2 per pair, already trimmed. */
int eo_scalar_map_pairs(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                        uint32_t n_pairs, const uint8_t* ref_codes, const uint64_t* ref_off,
                        const uint32_t* ref_len, uint32_t n_refs, int32_t ma, int32_t mi,
                        int32_t o, int32_t e, int both_strands, int local, int32_t min_score,
                        int threads, uint32_t cap, eo_pair_result* results, uint32_t* ties);

/* ---- traceback (scalar.rs:182-364) ---------------------------------- */
typedef struct eo_alignment {
    int32_t score;
    uint32_t query_start, query_end; /* 0-based, half-open */
    uint32_t ref_start, ref_end;
    uint32_t n_ops;                  /* BAM CIGAR words written */
} eo_alignment;

/* The best alignment's score, coordinates and ops (len << 4 | M=0 I=1 D=2).
 * Returns 0, -1 out of memory, -2 ops_cap too small.  n or m empty, or a
 * local alignment with no positive cell: all zero. */
int eo_align(const uint8_t* q, size_t n, const uint8_t* r, size_t m, int32_t ma, int32_t mi,
             int32_t o, int32_t e, int local, eo_alignment* out, uint32_t* ops, size_t ops_cap);
/* eo_align over a batch of jobs on OpenMP threads (the timed CPU baseline);
 * returns the thread count, -1 if an ops stride was too small. */
int eo_align_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                   const uint8_t* ref_codes, const uint64_t* ref_off, const uint32_t* ref_len,
                   const uint32_t* job_read, const uint32_t* job_ref, const uint8_t* job_rev,
                   uint32_t n_jobs, int32_t ma, int32_t mi, int32_t o, int32_t e, int local,
                   int threads, eo_alignment* out, uint32_t* ops, size_t ops_stride);

/* ---- MD / NM (sam.rs:55-121) ---------------------------------------- */
/* md_nm on codes: a base matches when both codes are equal and below 4
 * (calmd_match, sam.rs:63-69, after alphabet.rs:29-50 folds case and U);
 * reference letters go into MD upper-cased from `ref_letters` (the reference
 * as in the FASTA), or as A/C/G/T/N from the codes when it is NULL.  The
 * read is `q` (n codes) as sequenced, aligned reverse-complemented when
 * `reverse`.  Writes at most md_cap characters (no terminator); returns the
 * MD length, or -1 if md_cap was too small. */
long eo_md_nm(const uint8_t* q, size_t n, int reverse, const uint8_t* ref_codes,
              const uint8_t* ref_letters, const eo_alignment* a, const uint32_t* ops, char* md,
              size_t md_cap, uint32_t* nm);
/* eo_md_nm over a batch of traced jobs on OpenMP threads (job k's ops at
 * ops + k * ops_stride, its MD at md + k * md_stride); returns the thread
 * count, -1 if an MD stride was too small. */
int eo_md_nm_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                   const uint8_t* ref_codes, const uint64_t* ref_off, const uint8_t* ref_letters,
                   const uint32_t* job_read, const uint32_t* job_ref, const uint8_t* job_rev,
                   const eo_alignment* al, const uint32_t* ops, size_t ops_stride,
                   uint32_t n_jobs, int threads, char* md, size_t md_stride, uint32_t* md_len,
                   uint32_t* nm);

#ifdef __cplusplus
}
#endif
#endif
