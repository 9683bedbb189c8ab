/*
 * eschalign_b200.h -- C ABI of the B200 panel scorer.
 *
 * Scores every read of a batch against every reference of a panel with the
 * Gotoh affine-gap recurrence (local or semi-global), on the forward strand
 * and optionally the reverse complement, and reduces each read on the device
 * to its best score, suboptimal score (SAM XS) and tie set.
 *
 * This is the boundary eschalign's `--device gpu` path calls in place of the
 * Rust `eschalign::cuda::GpuScorer` (crates/eschalign/src/cuda/mod.rs:328-709).
 * Every entry point cites the reference interface it replaces.  Inputs are
 * alphabet codes (0..3 = A,C,G,T; 4 = any other letter, a wildcard that
 * matches everything), exactly what GpuScorer::score_batch takes
 * (cuda/mod.rs:524).  Plain pointers and sizes only; the library owns all
 * device memory; a scorer is used by one thread at a time, like GpuScorer
 * (`&mut self`, cuda/mod.rs:326-327), while different scorers, each on its
 * own stream, may be used from different threads at once.
 */
#ifndef ESCHALIGN_B200_H
#define ESCHALIGN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESG_ABI_VERSION 1

/* ---- status codes: GpuError (cuda/mod.rs:144-153) + AlignError (error.rs:7-28) */
typedef int32_t esg_status;
#define ESG_OK 0
#define ESG_ERR_UNAVAILABLE 1        /* GpuError::Unavailable: no driver or no device   */
#define ESG_ERR_DRIVER 2             /* GpuError::Driver: a CUDA call failed             */
#define ESG_ERR_REFERENCE_TOO_LONG 3 /* GpuError::ReferenceTooLong                       */
#define ESG_ERR_SCORING_INVALID 4    /* AlignError::ScoringInvalid (scoring.rs:70-100)   */
#define ESG_ERR_EMPTY_PANEL 5        /* AlignError::EmptyPanel (panel.rs:264-266)        */
#define ESG_ERR_EMPTY_REFERENCE 6    /* AlignError::EmptyReference (panel.rs:257-259)    */
#define ESG_ERR_BAD_ARGUMENT 7       /* a NULL pointer, a bad flag, a mode out of range  */
#define ESG_ERR_OUT_OF_MEMORY 8      /* device or pinned memory exhausted                */
#define ESG_ERR_TIMEOUT 9            /* a bounded device wait gave up                    */

/* ---- scoring: Scoring (scoring.rs:27-36) and Mode (scoring.rs:151-165) */
typedef struct esg_scoring {
    int32_t match_score; /* > 0                                   */
    int32_t mismatch;    /* < match_score                         */
    int32_t gap_open;    /* whole cost of a one-base gap, <= 0    */
    int32_t gap_extend;  /* each further base of the same gap, <= 0 */
} esg_scoring;

#define ESG_MODE_LOCAL 0
#define ESG_MODE_SEMIGLOBAL 1

/* ---- kernel choice: the A/B lever of GpuScorer::set_half2 (cuda/mod.rs:500) */
#define ESG_KERNEL_AUTO 0    /* batched int16x2 kernel, int32 lanes for what it cannot take */
#define ESG_KERNEL_PLAIN32 1 /* every query in int32, one thread per (query, reference)     */
#define ESG_KERNEL_INT32 2   /* every query on the int32 lanes (up to 32 lanes a reference) */

/* ---- batch flags */
#define ESG_BOTH_STRANDS 1u /* also score each read's reverse complement (align.rs:2865-2872) */
#define ESG_FULL_ROWS 2u    /* also return every query's scores (ScoreMatrix, mapper.rs:95-139) */

/* ---- per-read result: the scored half of Aligner::map_reads_scored
 * (mapper.rs:444-472).  Candidates are (reference r, strand) in the order
 * r = 0.. in panel order, forward before reverse; a candidate is written as
 * (r << 1) | reverse. */
typedef struct esg_read_result {
    int32_t best;       /* max over the read's candidates                        */
    int32_t suboptimal; /* max over candidates != best (XS); ESG_NO_SCORE if none */
    uint32_t n_tied;    /* how many candidates score `best`, counted in full     */
    uint32_t flags;     /* ESG_RESULT_* */
} esg_read_result;

#define ESG_NO_SCORE INT32_MIN
#define ESG_NO_TIE 0xffffffffu       /* tie-list slots past min(n_tied, tie_capacity)  */
#define ESG_RESULT_EMPTY 1u          /* empty read: no candidates (best = ESG_NO_SCORE) */
#define ESG_RESULT_TIES_TRUNCATED 2u /* n_tied > tie_capacity: only the first listed    */
#define ESG_RESULT_RESCORED32 4u     /* some pair was (re)scored by the int32 kernel    */

#define ESG_MAX_TIE_CAPACITY 32

typedef struct esg_options {
    uint32_t tie_capacity; /* ties listed per read, 1..ESG_MAX_TIE_CAPACITY (default 8)  */
    int32_t kernel;        /* ESG_KERNEL_*                                                */
    void* stream;          /* cudaStream_t to run on; NULL: the scorer makes its own      */
} esg_options;

typedef struct esg_info {
    char device_name[256]; /* GpuScorer::device_name (cuda/mod.rs:446)                */
    int32_t device;
    int32_t sm_count;
    uint32_t n_refs;
    uint32_t max_ref_len;
    uint32_t n_ref_pairs;     /* references paired into int16x2 lanes               */
    uint32_t panel_bytes;     /* shared-memory panel staged per CTA (0: read from L2) */
    int32_t batched_ok;       /* the scoring scheme fits the batched kernel's tables  */
    int32_t regs_batched;     /* GpuScorer::registers analogue (cuda/mod.rs:466)      */
    int32_t regs_plain;
    int32_t local_bytes_batched; /* GpuScorer::local_bytes analogue (cuda/mod.rs:479) */
    int32_t local_bytes_plain;
    int32_t batched_blocks;   /* persistent CTAs of the batched kernel                 */
    int32_t batched_threads;  /* threads per CTA                                       */
    int32_t plain_blocks;
    int32_t plain_threads;
    uint32_t split_len;       /* queries up to this length take 16-row stripes  */
    int32_t tuned;            /* split_len was measured by esg_scorer_autotune   */
} esg_info;

/* What esg_scorer_autotune measured (device time of calibration batches
 * cut from this panel) and chose.  Scores do not depend on any choice. */
#define ESG_TUNE_MAX_LENGTHS 8
typedef struct esg_tune_report {
    uint32_t n_lengths;
    uint32_t lengths[ESG_TUNE_MAX_LENGTHS];   /* read lengths (each batch +-25 %)      */
    float ms_rows16[ESG_TUNE_MAX_LENGTHS];    /* batched kernel, 16-row stripes        */
    float ms_rows32[ESG_TUNE_MAX_LENGTHS];    /* batched kernel, 32-row stripes        */
    uint32_t split_len;                       /* chosen: 16-row stripes up to this     */
    float ms_int32[ESG_TUNE_MAX_LENGTHS];     /* every query on the int32 lanes        */
    uint32_t int32_from;                      /* chosen: int32 lanes from this length (0: never) */
    uint32_t n_ctas16;                        /* resident CTAs per SM tried, 16-row tiles */
    uint32_t cand_ctas16[4];
    float ms_ctas16[4];
    uint32_t ctas16;                          /* chosen                                 */
    uint32_t n_ctas32;                        /* the same for 32-row tiles              */
    uint32_t cand_ctas32[4];
    float ms_ctas32[4];
    uint32_t ctas32;
    uint32_t n_chunk_targets;                 /* panel-chunk targets tried (tasks per resident warp) */
    uint32_t chunk_targets[8];
    float ms_chunks[8];
    uint32_t chunk_target;                    /* chosen                                 */
    uint32_t n_splits;                        /* esg_scorer_autotune_lengths: 16/32 splits tried */
    uint32_t splits[8];                       /* on one batch of the given length histogram */
    float ms_splits[8];
} esg_tune_report;

typedef struct esg_batch_stats {
    uint32_t n_reads;
    uint32_t n_queries;         /* reads x strands                                     */
    uint32_t n_empty;
    uint32_t queries_batched;   /* on the int16x2 kernel                               */
    uint32_t queries_plain;     /* put on the int32 kernel by the host                 */
    uint32_t queries_rescored;  /* flagged by the int16x2 kernel, re-scored in int32   */
    uint32_t tasks;             /* 32-lane work tiles of the batched kernel            */
    uint32_t lanes_used;        /* of tasks * 32                                       */
    uint32_t kernels;           /* kernels one launch of the batch runs                */
    uint64_t cells;             /* sum over scored queries of len * panel bases        */
    uint64_t h2d_bytes;
    uint64_t d2h_bytes;
    uint32_t n_pairs;           /* paired batches: read pairs (n_reads / 2)           */
    uint32_t mates_trimmed;     /* mates with an adapter found                         */
    uint64_t bases_trimmed;     /* adapter bases removed                               */
    uint32_t panel_chunks;      /* reference-pair chunks per tile (1: whole panel)     */
    uint32_t reserved;
    uint64_t device_bytes;      /* device memory the batch takes while submitted       */
} esg_batch_stats;

typedef struct esg_scorer esg_scorer;
typedef struct esg_batch esg_batch;

int esg_abi_version(void);
const char* esg_status_string(esg_status status);
/* Message of the last failure on this thread ("" if none). */
const char* esg_last_error(void);

/* device_visible (cuda/mod.rs:130-140): number of CUDA devices, 0 if none. */
esg_status esg_device_count(int32_t* out);

/* fits_i16 (crates/eschalign/src/simd/mod.rs:222-227): whether the reference's
 * SIMD kernels score a read of `len` bases; the reference GPU scorer's
 * scores_len (cuda/mod.rs:506-508) also requires 0 < len <= 4096.  This
 * scorer scores every non-empty read whatever this says. */
int32_t esg_fits_i16(uint64_t len, uint64_t max_ref_len, const esg_scoring* scoring);

/* GpuScorer::new_on_device (cuda/mod.rs:350-443): lay `n_refs` references
 * (codes, concatenated; reference r is ref_codes[ref_off[r] .. +ref_len[r]])
 * out on device `device` under one scoring and mode.  Refuses an invalid
 * scheme, an empty panel or reference, or a reference longer than 32768. */
esg_status esg_scorer_new(int32_t device, const uint8_t* ref_codes, const uint64_t* ref_off,
                          const uint32_t* ref_len, uint32_t n_refs, const esg_scoring* scoring,
                          int32_t mode, const esg_options* options, esg_scorer** out);
/* Frees the scorer and the device memory its batches used: batches take
 * their device memory from a pool the scorer owns, which keeps what a freed
 * batch returns for the next one (device memory in use grows to the largest
 * set of batches alive at once and is returned here).  Free every batch
 * first. */
void esg_scorer_free(esg_scorer* scorer);

esg_status esg_scorer_info(const esg_scorer* scorer, esg_info* out);
/* GpuScorer::set_half2 (cuda/mod.rs:500-502): ESG_KERNEL_AUTO, _PLAIN32 or
 * _INT32.  Choosing _PLAIN32 the first time makes its column buffers
 * (32 x max_ref_len x 8 bytes per warp, at most 1 GiB). */
esg_status esg_scorer_set_kernel(esg_scorer* scorer, int32_t kernel);
/* Tile-shape autotuner (no counterpart in the reference, whose one kernel
 * shape is fixed, cuda/mod.rs:238-301).  On calibration batches cut from
 * this panel (read lengths 48..448, each +-25 %) it times the batched kernel
 * with 16-row and with 32-row stripes and every query on the int32 lanes,
 * and sets the length up to which 16-row stripes are used and the length
 * from which queries go to the int32 lanes (where the batched kernel would
 * flag most of them); then the resident CTAs per SM of the 16- and 32-row
 * tiles (the occupancy limit and one or two fewer) and the panel-chunk
 * target for batches too small to fill the GPU.  Scores do not depend on
 * the choices.  `out` may be NULL. */
esg_status esg_scorer_autotune(esg_scorer* scorer, esg_tune_report* out);
/* The same, for a workload whose read lengths are sampled in `lens` (n of
 * them; zeros ignored): the 16/32-row split is then chosen on one
 * calibration batch drawn from that length histogram, every candidate split
 * (0, 48, ..., 512) timed on it, the fastest kept (the per-length
 * measurements still set the int32 lanes' length).  No counterpart in the
 * reference. */
esg_status esg_scorer_autotune_lengths(esg_scorer* scorer, const uint32_t* lens, uint32_t n,
                                       esg_tune_report* out);
/* Set the 16/32-row split by hand (0: every query on 32-row stripes). */
esg_status esg_scorer_set_split(esg_scorer* scorer, uint32_t split_len);

/* Panel chunking (no counterpart in the reference): when a batch has too
 * few 32-lane tiles to keep every resident warp busy to the end (few reads,
 * or a large panel), each tile's reference pairs are cut into up to
 * `max_chunks` chunks of about equal columns, one task each, and the
 * per-chunk states are merged on the device.  1 turns it off; default 64.
 * Scores do not depend on it. */
esg_status esg_scorer_set_chunking(esg_scorer* scorer, uint32_t max_chunks);

/* GpuScorer::scores_len (cuda/mod.rs:506-508): 1 for every len > 0 -- nothing
 * is left to a CPU path. */
int32_t esg_scores_len(const esg_scorer* scorer, uint64_t len);
/* GpuScorer::half2_scores_len (cuda/mod.rs:509-514), the fast kernel's
 * share: 1 when a query of `len` bases goes to the batched int16x2 kernel
 * (ESG_KERNEL_AUTO; in semi-global mode while its gap floor
 * 2 |open| + (min(len, longest reference) - 1) |extend| stays under 15000),
 * 0 when it goes to the int32 lanes.  A query the batched kernel takes may
 * still be flagged there and re-scored in int32. */
int32_t esg_batched_takes(const esg_scorer* scorer, uint64_t len);

/* GpuScorer::score_batch (cuda/mod.rs:524-528): prepare + submit + finish.
 * Read k is codes[off[k] .. off[k] + len[k]].  `results` gets n_reads
 * entries, `ties` n_reads * tie_capacity candidates (first n_listed of each
 * read are valid, n_listed = min(n_tied, tie_capacity)).  With
 * ESG_FULL_ROWS, `rows` gets every query's scores in panel order, forward
 * rows 0..n_reads-1 then (ESG_BOTH_STRANDS) reverse rows n_reads..2n-1 --
 * the reference's batch layout (align.rs:1484-1494); an empty read's rows
 * are 0, the score of an empty query (scalar.rs:120-163). */
esg_status esg_score_batch(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_reads, uint32_t flags,
                           esg_read_result* results, uint32_t* ties, int32_t* rows);

/* GpuScorer::prepare (cuda/mod.rs:533-576): host only, touches no device
 * state, so it may run while an earlier batch's kernels do.  Copies the
 * reads into pinned staging and plans the work (length buckets, 32-lane
 * tiles, int32 list). */
esg_status esg_prepare(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                       const uint32_t* len, uint32_t n_reads, uint32_t flags, esg_batch** out);
/* GpuScorer::submit (cuda/mod.rs:581-699): upload and queue the kernels on
 * the scorer's stream; returns without waiting. */
esg_status esg_submit(esg_scorer* scorer, esg_batch* batch);
/* GpuScorer::finish (cuda/mod.rs:702-708): wait for the batch and copy its
 * results to the caller's buffers (any of ties/rows may be NULL). */
esg_status esg_finish(esg_scorer* scorer, esg_batch* batch, esg_read_result* results,
                      uint32_t* ties, int32_t* rows);
void esg_batch_free(esg_batch* batch);
esg_status esg_batch_stats_get(const esg_batch* batch, esg_batch_stats* out);

/* Re-run the device work of a submitted batch on `stream` (NULL: the
 * scorer's) with its inputs already resident, no copies.  For measuring the
 * kernels alone; the batch's results are overwritten with identical ones. */
esg_status esg_relaunch(esg_scorer* scorer, esg_batch* batch, void* stream);
/* A batch's device work (counter reset, the batched kernel's three task
 * groups on two streams, the chunk merge, the int32 path, the per-read
 * merge, the pair ranking) is captured once as a CUDA graph at esg_submit
 * and launched as one graph, by esg_submit and esg_relaunch; the scorer
 * keeps one instantiated graph per launch-sequence shape and updates it
 * with each batch's parameters.  No counterpart in the reference, which
 * launches its kernels one by one (cuda/mod.rs:581-699).  enabled = 0
 * launches the kernels one by one instead; results are the same.  A
 * scorer whose stream the caller is capturing launches one by one. */
esg_status esg_scorer_set_graphs(esg_scorer* scorer, int32_t enabled);
/* Copy a submitted batch's per-read results and ties as they stand in device
 * memory now -- after esg_relaunch, the last launch's -- into the caller's
 * buffers (ties may be NULL), after the device has finished its work.  No
 * counterpart in the reference: it checks that relaunched work, the work a
 * benchmark times, gives the results esg_finish returned. */
esg_status esg_batch_read_results(esg_scorer* scorer, esg_batch* batch, esg_read_result* results,
                                  uint32_t* ties);

/* ---- paired-end: the scored half of Aligner::map_pairs_scored
 * (crates/eschalign/src/mapper/pair.rs:157-234) fed the way the CLI's GPU
 * thread feeds it (crates/eschalign-cli/src/align.rs:2844-2872): mates
 * trimmed of their 3' adapter (adapter.rs:68-110, align.rs:934-949), each
 * mate scored as sequenced and reverse-complemented, and the candidates
 * (reference, template strand) ranked on the device. */

/* AdapterConfig (adapter.rs:46-54) plus the CLI's --max-read-len.  Adapters
 * are codes (alphabet.rs); r1_len = r2_len = 0 trims nothing. */
typedef struct esg_adapter_config {
    const uint8_t* r1;     /* adapter prefix on mate 1's 3' end (TRUSEQ_R1, adapter.rs:40) */
    uint32_t r1_len;
    const uint8_t* r2;     /* on mate 2's (TRUSEQ_R2, adapter.rs:42)                        */
    uint32_t r2_len;
    uint32_t min_overlap;  /* DEFAULT_MIN_OVERLAP = 5 (adapter.rs:44); 0 counts as 1       */
    uint32_t max_read_len; /* a longer mate is not aligned nor searched; 0 = no limit      */
} esg_adapter_config;

/* pair_adapters (crates/eschalign-cli/src/align.rs:934-949) over a batch,
 * host only (no device needed): mates 2p and 2p + 1; adapter_bases[2n] gets
 * each mate's adapter bases, aligned_len[2n] the bases left to align (0 for
 * a mate over max_read_len, align.rs:2851-2853).  esg_prepare_pairs trims
 * with this same code. */
esg_status esg_pair_adapters(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                             uint32_t n_pairs, const esg_adapter_config* adapters,
                             uint32_t* adapter_bases, uint32_t* aligned_len);

/* One pair's ranked candidates (pair.rs:195-234).  Candidate (r, t): t = 0
 * mate 1 as sequenced + mate 2 reverse-complemented, t = 1 the opposite;
 * eligible when both mate scores are >= min_score; ranked by (-sum, r, t).
 * The first tier is the tie set the reference traces first; `next` lets it
 * fall through without rescoring.  `xs` is PairMapping::Proper's per-mate
 * suboptimal (pair.rs:297-314) for a pair whose whole first tier passes the
 * pair constraints.  No eligible candidate (or an empty mate):
 * ESG_RESULT_EMPTY, and the per-mate read results are the Separate fallback
 * (pair.rs:366-387). */
typedef struct esg_pair_result {
    int32_t best;       /* first tier's summed score; ESG_NO_SCORE if no candidate */
    int32_t next;       /* the next tier's sum; ESG_NO_SCORE if none                */
    uint32_t n_tied;    /* candidates in the first tier, counted in full            */
    uint32_t flags;     /* ESG_RESULT_EMPTY / _TIES_TRUNCATED / _RESCORED32         */
    int32_t xs[2];      /* per mate: best score over candidates outside the tier   */
    int32_t primary[2]; /* the first tie's two mate scores                          */
} esg_pair_result;

/* Pair flag for esg_prepare_pairs: ESG_BOTH_STRANDS ranks both template
 * strands (PairOptions::both_strands, pair.rs:52); ESG_FULL_ROWS returns the
 * four rows per pair. */
/* Plan a paired batch: mates are reads 2p (mate 1) and 2p + 1 (mate 2) of
 * codes/off/len (as sequenced).  Trims them (host threads) per `adapters`
 * (NULL: no trimming), then plans every mate on both strands.  Submit and
 * relaunch as any batch. */
esg_status esg_prepare_pairs(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                             const uint32_t* len, uint32_t n_pairs,
                             const esg_adapter_config* adapters, int32_t min_score,
                             uint32_t flags, esg_batch** out);
/* Wait for a paired batch and copy out (any pointer may be NULL):
 *   pairs[n_pairs], pair_ties[n_pairs * tie_capacity] as (ref << 1) | t;
 *   mates[2 n_pairs], mate_ties[2 n_pairs * tie_capacity]: each mate alone on
 *     both strands, as map_reads_scored ranks it (mapper.rs:444-472);
 *   adapters[2 n_pairs]: adapter bases removed from each mate;
 *   rows[4 n_pairs * n_refs] (ESG_FULL_ROWS): forward rows of the 2 n_pairs
 *     mates, then their reverse-complement rows. */
esg_status esg_finish_pairs(esg_scorer* scorer, esg_batch* batch, esg_pair_result* pairs,
                            uint32_t* pair_ties, esg_read_result* mates, uint32_t* mate_ties,
                            uint32_t* adapters, int32_t* rows);
/* prepare_pairs + submit + finish_pairs. */
esg_status esg_score_pairs(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_pairs,
                           const esg_adapter_config* adapters, int32_t min_score, uint32_t flags,
                           esg_pair_result* pairs, uint32_t* pair_ties, esg_read_result* mates,
                           uint32_t* mate_ties, uint32_t* adapter_bases, int32_t* rows);

/* Merge two sets of per-read results over disjoint candidate sets (e.g. two
 * panel shards; candidate numbers global, (ref << 1) | reverse) into the
 * result over their union, as mapper.rs:444-472 would give it: the higher
 * best wins, equal bests add their tie counts and merge their lists in
 * candidate order, XS is the best score outside the union's tie set.  Host
 * only.  `out`/`out_ties` may alias `a`/`a_ties`. */
esg_status esg_merge_read_results(const esg_read_result* a, const uint32_t* a_ties,
                                  const esg_read_result* b, const uint32_t* b_ties,
                                  uint32_t n_reads, uint32_t tie_capacity, esg_read_result* out,
                                  uint32_t* out_ties);

/* ---- traceback of winners: scalar::align (crates/eschalign/src/scalar.rs:
 * 182-364), the alignment eschalign traces for each read's tie set after
 * scoring (mapper.rs:494-495 -> simd::align_pairs, simd/mod.rs:405-499).
 * Same end cell (the first maximum of a column-major scan), same path
 * (diagonal, then insertion, then deletion; extending inside a gap; local
 * mode stops at the first zero cell). */
typedef struct esg_align_job {
    uint32_t read;     /* read index in the batch                         */
    uint32_t ref;      /* reference, panel order                          */
    uint32_t reverse;  /* 1: align the read's reverse complement          */
} esg_align_job;

/* One traced alignment.  Coordinates 0-based, half-open; ops are BAM CIGAR
 * words (len << 4 | op; M = 0, I = 1, D = 2), ops[ops_offset ..
 * ops_offset + n_ops), first to last.  A local alignment with no positive
 * cell is all zero (scalar.rs:81-85). */
typedef struct esg_alignment {
    int32_t score;
    uint32_t query_start, query_end;
    uint32_t ref_start, ref_end;
    uint32_t n_ops;
    uint64_t ops_offset;
} esg_alignment;

/* Trace `jobs` against the reads of a submitted batch (its reads are still
 * on the device: call after esg_finish, before esg_batch_free).  `ops`
 * holds ops_capacity words; ESG_ERR_BAD_ARGUMENT if the alignments need
 * more (the needed count is then in *ops_needed, which may be NULL). */
esg_status esg_align_batch(esg_scorer* scorer, esg_batch* batch, const esg_align_job* jobs,
                           uint32_t n_jobs, esg_alignment* out, uint32_t* ops,
                           uint64_t ops_capacity, uint64_t* ops_needed);
/* The same for reads given here (uploaded, then traced). */
esg_status esg_align_reads(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                           const uint32_t* len, uint32_t n_reads, const esg_align_job* jobs,
                           uint32_t n_jobs, esg_alignment* out, uint32_t* ops,
                           uint64_t ops_capacity, uint64_t* ops_needed);

/* ---- mapping: Aligner::map_reads_scored (crates/eschalign/src/mapper.rs:
 * 400-552) fed by this scorer's fused reduction instead of a ScoreMatrix.
 * Every read is scored against the panel (its reverse complement too with
 * both_strands), its tie set taken in candidate order -- the first
 * min(n_tied, max_ties + 1) members, none below min_score -- and each taken
 * member traced on the device (esg_align_batch); the read is unmapped when
 * it takes none or its primary traces to no aligned base (a local score of
 * zero).  Reads whose taken ties outrun the scorer's tie capacity are scored
 * again with full rows for the rest of their list.  Each hit carries MD and
 * NM as samtools calmd writes them (sam.rs:71-121): a base matches only when
 * both are A/C/G/T (U as T) and equal; mismatched and deleted reference
 * letters are written upper-cased from `ref_letters` (panel letters, reference
 * r at ref_letters[ref_letter_off[r] .. + its length]), or, when that is
 * NULL, as A/C/G/T/N from the panel's codes. */
#define ESG_ALL_TIES 0xffffffffu /* MapOptions::max_ties = None: trace every tie */

typedef struct esg_map_options {   /* MapOptions (mapper.rs:32-40)                   */
    int32_t min_score;             /* a read whose best is below this is unmapped    */
    uint32_t max_ties;             /* ties traced besides the primary; ESG_ALL_TIES  */
    uint32_t both_strands;         /* also score and trace the reverse complement    */
    uint32_t reserved;             /* 0                                              */
} esg_map_options;

#define ESG_MAPPING_HAS_BEST 1u       /* best_score is set (the read is not empty) */
#define ESG_MAPPING_HAS_SUBOPTIMAL 2u /* suboptimal is set (not every candidate ties) */

typedef struct esg_read_mapping {  /* ReadMapping (mapper.rs:60-70)                    */
    int32_t best_score;
    int32_t suboptimal;            /* SAM XS                                          */
    uint32_t n_tied;
    uint32_t flags;                /* ESG_MAPPING_*                                   */
    uint32_t n_hits;               /* primary first, then the other taken ties; 0 = unmapped */
    uint32_t reserved;
    uint64_t first_hit;            /* this read's hits: hits[first_hit .. + n_hits)    */
} esg_read_mapping;

typedef struct esg_hit {           /* Hit (mapper.rs:43-56)                            */
    uint32_t reference;            /* panel order                                     */
    uint32_t reverse;              /* the read's reverse complement aligned           */
    esg_alignment alignment;       /* coordinates on the read as aligned; ops in esg_mapping_ops */
    uint32_t nm;
    uint32_t md_len;
    uint64_t md_offset;            /* MD at md[md_offset .. + md_len), not NUL-terminated */
} esg_hit;

typedef struct esg_mapping esg_mapping;

esg_status esg_map_reads(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                         const uint32_t* len, uint32_t n_reads, const esg_map_options* options,
                         const uint8_t* ref_letters, const uint64_t* ref_letter_off,
                         esg_mapping** out);
/* ---- paired mapping: Aligner::map_pairs_scored (crates/eschalign/src/
 * mapper/pair.rs:157-390) over the device ranking.  Mates 2p and 2p + 1 are
 * pair p as given (trim adapters first, esg_pair_adapters, as the CLI does
 * before map_pairs_scored).  Each pair's eligible candidates (reference,
 * template strand) are taken tier by tier in descending summed score; the
 * first tier with members whose traced mates satisfy the pair constraints
 * (both aligned, no outie, insert <= max_insert; pair.rs:392-410) is the tie
 * set, XS per mate is the best mate score outside it, and a pair with no
 * such tier maps each mate on its own, both strands, as esg_map_reads
 * does.  The first tier comes from the device ranking; deeper tiers, and a
 * first tier longer than the tie capacity, from full rows. */
typedef struct esg_pair_map_options { /* PairOptions (pair.rs:44-65)                  */
    int32_t min_score;            /* both mates at least this                        */
    uint32_t max_ties;            /* pair hits besides the primary; ESG_ALL_TIES     */
    uint32_t max_insert;          /* longest insert, bases (the reference's default 500) */
    uint32_t both_strands;        /* also the reverse template strand                */
} esg_pair_map_options;

#define ESG_PAIR_PROPER 1u  /* PairMapping::Proper; else Separate: the mates in esg_mapping_reads */
#define ESG_PAIR_HAS_XS1 2u /* suboptimal[0] is set                                            */
#define ESG_PAIR_HAS_XS2 4u /* suboptimal[1] is set                                            */

typedef struct esg_pair_mapping { /* PairMapping (pair.rs:89-105)                       */
    uint32_t flags;               /* ESG_PAIR_*                                          */
    int32_t score;                /* Proper: the pair score (both mates summed)          */
    uint32_t n_tied;              /* Proper: the tie set's size                          */
    uint32_t n_hits;              /* Proper: primary first, then up to max_ties more     */
    int32_t suboptimal[2];        /* Proper: per mate XS                                 */
    uint64_t first_hit;           /* Proper: pair_hits[first_hit .. + n_hits)            */
} esg_pair_mapping;

typedef struct esg_pair_hit {     /* PairHit (pair.rs:68-81)                             */
    uint32_t reference;           /* panel order                                         */
    uint32_t reverse;             /* template on the reverse strand                      */
    uint64_t insert;              /* leftmost aligned reference base to rightmost        */
    esg_hit mates[2];             /* each mate's own strand; coordinates on it as aligned */
} esg_pair_hit;

esg_status esg_map_pairs(esg_scorer* scorer, const uint8_t* codes, const uint64_t* off,
                         const uint32_t* len, uint32_t n_pairs,
                         const esg_pair_map_options* options, const uint8_t* ref_letters,
                         const uint64_t* ref_letter_off, esg_mapping** out);
/* A paired mapping's pairs and pair hits; its esg_mapping_reads holds the
 * two mates of each pair (2p, 2p + 1), filled for Separate pairs. */
const esg_pair_mapping* esg_mapping_pairs(const esg_mapping* mapping, uint32_t* n);
const esg_pair_hit* esg_mapping_pair_hits(const esg_mapping* mapping, uint64_t* n);

/* The arrays of a mapping (owned by it; valid until esg_mapping_free). */
const esg_read_mapping* esg_mapping_reads(const esg_mapping* mapping, uint32_t* n);
const esg_hit* esg_mapping_hits(const esg_mapping* mapping, uint64_t* n);
const uint32_t* esg_mapping_ops(const esg_mapping* mapping, uint64_t* n);
const char* esg_mapping_md(const esg_mapping* mapping, uint64_t* n);
void esg_mapping_free(esg_mapping* mapping);
/* A mapping made from the caller's arrays (copied; the same layout the
 * accessors above return), for reads mapped elsewhere that go to
 * esg_bam_encode.  Offsets are checked against the arrays, and each hit
 * must be one a traceback gives: strand 0 or 1, each start at most its end,
 * CIGAR words of the BAM ops M..X whose read- and reference-consuming
 * lengths span [query_start, query_end) and [ref_start, ref_end); anything
 * else is ESG_ERR_BAD_ARGUMENT naming the hit.  No counterpart in the
 * reference. */
esg_status esg_mapping_from_arrays(const esg_read_mapping* reads, uint32_t n_reads,
                                   const esg_hit* hits, uint64_t n_hits, const uint32_t* ops,
                                   uint64_t n_ops, const char* md, uint64_t n_md,
                                   esg_mapping** out);
/* Give a mapping made by esg_mapping_from_arrays the paired arrays of
 * esg_map_pairs' output (two read entries per pair; offsets and each mate's
 * hit checked as above), for esg_bam_encode_pairs. */
esg_status esg_mapping_set_pairs(esg_mapping* mapping, const esg_pair_mapping* pairs,
                                 uint32_t n_pairs, const esg_pair_hit* pair_hits,
                                 uint64_t n_pair_hits);

/* ---- serving: a request queue over resident scorers.  No counterpart in
 * the reference, which scores batches of one stream of reads and has no
 * serving mode.  Requests name a scorer slot (a resident panel under one
 * scoring and mode) and a strand flag; each slot's worker thread batches
 * whatever requests of that slot are waiting (continuous batching: up to
 * max_batch_reads reads and max_batch_cells DP cells per batch -- a larger
 * request runs as several batches -- and max_inflight batches queued on the
 * scorer's stream) and admits a batch only when its device memory fits the
 * free device memory (cudaMemGetInfo, plus what the scorer's pool holds
 * spare) less a headroom, and the budget if one is set.  A request that can
 * never fit is refused with ESG_ERR_OUT_OF_MEMORY.  Results are the ones
 * esg_score_batch gives for the same reads alone. */
typedef struct esg_server esg_server;

typedef struct esg_server_options {
    uint32_t max_batch_reads;  /* reads per batch at most (0: 262144)                            */
    uint32_t max_inflight;     /* batches queued per scorer (0: 2)                               */
    uint64_t memory_budget;    /* device bytes of admitted batches at most (0: free memory only) */
    uint64_t memory_headroom;  /* device bytes admission leaves free (0: 256 MiB)                */
    uint64_t max_batch_cells;  /* DP cells per batch at most (0: 1.5e11, ~30 ms); a larger
                                  request is cut into pieces of whole reads                      */
} esg_server_options;

typedef struct esg_request_timing {
    double queued_ms;          /* submit -> its batch went to the device                         */
    double total_ms;           /* submit -> its results were ready                               */
    uint32_t batch_reads;      /* reads of the batch it rode in                                  */
    uint32_t batch_requests;   /* requests of that batch                                         */
} esg_request_timing;

typedef struct esg_server_stats {
    uint64_t requests;         /* submitted                                                      */
    uint64_t completed;        /* results ready (scored or failed)                               */
    uint64_t refused;          /* refused by admission (could never fit)                         */
    uint64_t batches;          /* batches run                                                    */
    uint64_t cells;            /* DP cells of the batches run                                    */
    uint64_t bytes_in_flight;  /* device bytes of admitted batches now                           */
    uint64_t peak_bytes_in_flight;
    uint32_t admission_waits;  /* times a batch waited for device memory                         */
    uint32_t kernels;          /* kernel launches of the batches run                             */
} esg_server_stats;

esg_status esg_server_new(const esg_server_options* options, esg_server** out);
/* Add a resident scorer as slot *slot (its worker starts).  The server does
 * not own the scorer: free the server first.  Use the scorer only through
 * the server afterwards. */
esg_status esg_server_add_scorer(esg_server* server, esg_scorer* scorer, uint32_t* slot);
/* Queue a request (thread-safe): the reads are copied, the caller's buffers
 * may be reused on return.  flags: 0 or ESG_BOTH_STRANDS. */
esg_status esg_server_submit(esg_server* server, uint32_t slot, const uint8_t* codes,
                             const uint64_t* off, const uint32_t* len, uint32_t n_reads,
                             uint32_t flags, uint64_t* ticket);
/* Wait up to timeout_ms (< 0: no limit; a host-side wait) for a request; on success copy its
 * results (n_reads entries) and ties (n_reads * tie_capacity; any pointer
 * may be NULL) and release the ticket.  ESG_ERR_TIMEOUT leaves the request
 * queued (wait again); any other error is the request's own status (its
 * ticket released). */
esg_status esg_server_wait(esg_server* server, uint64_t ticket, int32_t timeout_ms,
                           esg_read_result* results, uint32_t* ties, esg_request_timing* timing);
esg_status esg_server_stats_get(esg_server* server, esg_server_stats* out);
/* Stop: each worker finishes its batches on the device and fails the
 * requests still queued; then the workers are joined and the server freed.
 * Call it once no other thread is inside esg_server_submit / _wait;
 * requests nobody waited for are dropped. */
void esg_server_free(esg_server* server);

/* ---- BAM input and output around the mapping stage (host code, zlib).
 *
 * The CLI's I/O stage for unpaired reads (crates/eschalign-cli/src/align.rs):
 * read_batches (604-660), the records of a read's mapping (build_records,
 * 1084-1200; process_chunk's --max-read-len rule, 1504-1602), and the
 * ordered or coordinate-sorted writer (write_in_order, 2345-2400; the sort,
 * 2406-2450).  A batch's reads go to esg_map_reads as they come
 * (esg_bam_batch_reads); its mapping comes back to esg_bam_encode, whose
 * records are byte for byte the reference CLI's: input tags kept, NM / MD /
 * AS / XS / XA replaced, MAPQ 60 for a unique best and 0 otherwise, the
 * primary hit's CIGAR with soft clips, XA for the other taken ties, and with
 * `secondary` one record per further tie. */
typedef struct esg_bam_reader esg_bam_reader;
typedef struct esg_bam_batch esg_bam_batch;
typedef struct esg_bam_records esg_bam_records;
typedef struct esg_bam_writer esg_bam_writer;
typedef struct esg_bam_options {
    uint32_t secondary; /* --secondary: one SECONDARY record per further taken tie */
    uint32_t reserved;  /* 0 */
} esg_bam_options;

/* Open the CLI's unpaired input (align.rs:385-414): a BGZF-compressed BAM
 * (header read; threads: inflating threads, 0 = the host's cores), or a
 * FASTA or FASTQ file, plain or gzip, told apart by content.  FASTX records
 * come in as unmapped records with no header (align.rs:436-563: the name up
 * to the first blank, sequences upper-cased with U as T and other letters
 * outside the BAM alphabet as N, FASTQ qualities Phred + 33, FASTA ones
 * missing).  An uncompressed BAM is refused, as the CLI refuses it. */
esg_status esg_bam_open(const char* path, uint32_t threads, esg_bam_reader** out);
const char* esg_bam_header_text(const esg_bam_reader* reader, uint64_t* len);
/* Open the CLI's paired input (PairSource, align.rs:674-870): mate 1 and
 * mate 2 FASTA / FASTQ files (path2 given; record k of each is a pair), or
 * one file holding both mates (path2 NULL): an interleaved FASTA / FASTQ or
 * a BAM whose mates are adjacent records flagged 0x1 with one of 0x40 /
 * 0x80.  Mates share the pair's name, a trailing /1 or /2 dropped. */
esg_status esg_bam_open_pairs(const char* path1, const char* path2, uint32_t threads,
                              esg_bam_reader** out);
/* The next pairs of a paired reader, at most max_pairs: records 2p (mate 1)
 * and 2p + 1 (mate 2), their reads at full length in esg_bam_batch_reads
 * (esg_pair_adapters trims them, and leaves mates over --max-read-len out).
 * An orphan mate, mates whose names differ or a BAM record that is not a
 * mate is ESG_ERR_BAD_ARGUMENT naming the read.  0 pairs: the end. */
esg_status esg_bam_read_pair_batch(esg_bam_reader* reader, uint32_t max_pairs,
                                   esg_bam_batch** out);
/* --read-ids (load_read_ids, canonical_read_name: align.rs:572-601): keep
 * only the reads (or pairs, by the pair's name) named in the file at
 * `path`, one name per line (its first word; blank lines and lines starting
 * '#' skipped).  A name that is a UUID -- dashed, 32 hex digits, braced or
 * urn:uuid: -- matches any spelling of it.  A file with no name is
 * ESG_ERR_BAD_ARGUMENT. */
esg_status esg_bam_set_read_ids(esg_bam_reader* reader, const char* path);
/* What the reader dropped so far: secondary / supplementary input records,
 * and reads not in --read-ids (two per pair). */
esg_status esg_bam_reader_counts(const esg_bam_reader* reader, uint64_t* not_primary,
                                 uint64_t* filtered);
/* The next primary records, at most max_reads (secondary and supplementary
 * ones skipped; a record aligned to the reverse strand is refused with
 * ESG_ERR_BAD_ARGUMENT, as is a malformed FASTA / FASTQ record).  A batch of
 * 0 reads means the end of the file.
 * Reads over max_read_len (0 = no limit) get length 0 in
 * esg_bam_batch_reads, so the mapping stage leaves them unmapped. */
esg_status esg_bam_read_batch(esg_bam_reader* reader, uint32_t max_reads, uint32_t max_read_len,
                              esg_bam_batch** out);
/* The batch's reads as alphabet codes (0..3 = A,C,G,T; 4 = any other base),
 * for esg_map_reads; owned by the batch. */
esg_status esg_bam_batch_reads(const esg_bam_batch* batch, const uint8_t** codes,
                               const uint64_t** off, const uint32_t** len, uint32_t* n_reads);
void esg_bam_batch_free(esg_bam_batch* batch);
void esg_bam_close(esg_bam_reader* reader);
/* The output records of a batch from its mapping (esg_map_reads over
 * esg_bam_batch_reads, with the panel's letters for MD), encoded in the BAM
 * layout, in read order; ref_names in panel order.  A hit whose reference
 * is past ref_names, or whose read coordinates run past its read, is
 * ESG_ERR_BAD_ARGUMENT. */
esg_status esg_bam_encode(const esg_bam_batch* batch, const esg_mapping* mapping,
                          const esg_bam_options* options, const char* const* ref_names,
                          uint32_t n_refs, uint32_t threads, esg_bam_records** out);
/* The records of a batch of pairs from esg_map_pairs over its trimmed
 * mates (build_pair_records, align.rs:1238-1425, with process_pair_chunk's
 * placements, 1683-1713): mate 1, mate 2, then with `secondary` a pair of
 * 0x100 records per further tie-set member.  Flags 0x1 / 0x2 / 0x8 / 0x20 /
 * 0x40 / 0x80, mate reference and position, TLEN, MC, and each mate's
 * adapter bases soft-clipped at its 3' end and counted in `ad`
 * (adapter_bases[2n] from esg_pair_adapters; NULL under --no-adapter-trim:
 * no `ad` tag).  A Proper pair with no pair hit, or a hit running past its
 * mate (with the mate's adapter bases), is ESG_ERR_BAD_ARGUMENT. */
esg_status esg_bam_encode_pairs(const esg_bam_batch* batch, const esg_mapping* mapping,
                                const uint32_t* adapter_bases, const esg_bam_options* options,
                                const char* const* ref_names, uint32_t n_refs, uint32_t threads,
                                esg_bam_records** out);
const uint8_t* esg_bam_records_bytes(const esg_bam_records* records, uint64_t* n_bytes,
                                     uint32_t* n_records);
/* How the batch's reads (mates, for pairs) went, the CLI's run summary
 * (Outcome, align.rs:1077-1082, 2360-2372): a unique best, a tie, unmapped. */
esg_status esg_bam_records_outcomes(const esg_bam_records* records, uint64_t* unique,
                                    uint64_t* tied, uint64_t* unmapped);
void esg_bam_records_free(esg_bam_records* records);
/* A BGZF BAM writer: header, then the records of the chunks pushed, in the
 * order of their sequence numbers 0, 1, ... whatever order they arrive in;
 * with sort_coordinate, in coordinate order at close (reference, position,
 * reverse after forward, then input order; unmapped last).  Blocks are
 * deflated on `threads` host threads (0 = the host's cores). */
esg_status esg_bam_writer_open(const char* path, const char* header_text,
                               const char* const* ref_names, const uint32_t* ref_lens,
                               uint32_t n_refs, int32_t sort_coordinate, uint32_t threads,
                               esg_bam_writer** out);
esg_status esg_bam_writer_push(esg_bam_writer* writer, uint64_t seq,
                               const esg_bam_records* records);
/* Writes what is left (the sorted records), the end-of-file block, and
 * frees the writer. */
esg_status esg_bam_writer_close(esg_bam_writer* writer);
/* Deflate the writer's blocks on `device` from now on (a negative device:
 * on the host threads again).  No counterpart in the reference, whose writer
 * deflates on host threads (noodles' MultithreadedWriter, align.rs:2066).
 * One warp per 0xff00-byte block: greedy LZ77 over 2040-byte stripes, one
 * dynamic-Huffman DEFLATE block per BGZF block, an incompressible block
 * stored; the file is a valid BGZF BAM whose records are those of the host
 * writer (its compressed bytes differ).  Each push uploads its whole blocks
 * and returns while the device compresses them; they are written at the
 * next push or at close.  Uses about 270 KiB of device memory per block of
 * the largest push, and the device's CUDA stream of greatest priority. */
esg_status esg_bam_writer_use_device(esg_bam_writer* writer, int32_t device);
/* Blocks written by the device so far, and how many of them stored. */
esg_status esg_bam_writer_blocks(const esg_bam_writer* writer, uint64_t* blocks,
                                 uint64_t* stored);
/* The device compressor's steps run on the host, lane by lane, on one block
 * (1 <= n <= 0xff00 bytes) into `out` (65536 bytes, 4-byte aligned): the
 * length of the raw DEFLATE stream, 0xffffffff when the block is to be
 * stored, 0 on a bad argument.  For checking the steps without a device;
 * the writer does not call it. */
uint32_t esg_bgzf_deflate_host(const uint8_t* src, uint32_t n, uint8_t* out);
/* The compressor's Huffman code lengths on the host: freq[0, n) (2 <= n <=
 * 288) to lengths of at most `limit` (1..15) bits, every symbol with a
 * frequency coded and the code complete.  0, or -1 on a bad argument. */
int32_t esg_bgzf_code_lengths(const uint32_t* freq, uint32_t n, uint32_t limit, uint8_t* len);

/* Scoring for callers that cannot allocate.  No counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc when they need scores: a process whose
 * device memory belongs to a framework's caching allocator, which forbids
 * allocations behind its back (they fragment its pool and escape its
 * budget), or a real-time loop that must not enter the driver's allocator
 * after start-up (cudaMalloc and cudaFree can block and synchronize the
 * device).  They call this instead of a scorer: it allocates nothing, host
 * or device.  The caller passes device buffers: queries (codes 0..4, query
 * q is d_codes[d_off[q] .. +d_len[q]], scored as given, forward only),
 * references (d_ref_codes[d_ref_off[r] .. +d_ref_len[r]]) and the output
 * d_rows[q * n_refs + r] (int32, the scalar oracle's score of every pair,
 * scalar.rs:120-163).  It runs the int32 lanes kernel on `stream` (NULL: the
 * legacy default stream) and returns without waiting.
 *
 * The kernel's column buffer (a reference's bottom row carried between the
 * passes of a query longer than 512 bases) is a 16 MiB array held on every
 * GPU where the library's module is loaded, until the process exits.  It
 * limits references to ESG_NOALLOC_MAX_REF_LEN bases: `max_ref_len` above
 * that is refused with ESG_ERR_REFERENCE_TOO_LONG, and a reference longer
 * than the stated max_ref_len (any reference, when it is 0) scores
 * ESG_NO_SCORE.  Under lazy module loading (the CUDA default) the module,
 * and with it the array, is loaded on a device by the first call there,
 * which also looks up the array's device address on that device (the
 * device must be current) and keeps it for the life of the process: that
 * first call can fail with ESG_ERR_OUT_OF_MEMORY, and it should come before
 * any stream capture.  The kept address does not survive cudaDeviceReset:
 * do not call this on a device after resetting it.  Every call shares the
 * one array: calls whose kernels overlap on the GPU (other streams, other
 * threads) race and must be serialized by the caller.  Nothing in the array
 * needs to start at zero. */
#define ESG_NOALLOC_MAX_REF_LEN 8192
esg_status esg_score_rows_noalloc(const uint8_t* d_codes, const uint64_t* d_off,
                                  const uint32_t* d_len, uint32_t n_queries,
                                  const uint8_t* d_ref_codes, const uint32_t* d_ref_off,
                                  const uint32_t* d_ref_len, uint32_t n_refs,
                                  uint32_t max_ref_len, const esg_scoring* scoring, int32_t mode,
                                  int32_t* d_rows, void* stream);

#ifdef __cplusplus
}
#endif
#endif
