/*
 * esg_cpu_avx512.c -- restatement of eschalign's AVX-512BW score kernels, the
 * CPU baseline timed beside the GPU path.
 *
 * TEST INFRASTRUCTURE ONLY (see esg_oracle.h).  Follows:
 *   - Profile::from_codes          crates/eschalign/src/simd/mod.rs:292-331
 *   - Group::tprof                  crates/eschalign/src/simd/mod.rs:255-269
 *   - row-major kernel<LOCAL>       crates/eschalign/src/simd/avx512.rs:43-107
 *   - transposed<LOCAL>             crates/eschalign/src/simd/avx512.rs:278-354
 *   - dispatch (kernel_for)         crates/eschalign/src/mapper.rs:216-222,
 *                                   TRANSPOSED_MIN_READ_LEN simd/mod.rs:117,
 *                                   fits_i16 simd/mod.rs:222-227
 *   - per-read selection            crates/eschalign/src/mapper.rs:444-472
 *   - 64-read chunks over workers   crates/eschalign-cli/src/align.rs:1470-1473
 * One reference per i16 lane, 32 lanes per zmm; lanes hold references sorted
 * longest first; i16 with wrapping adds and NEG16 = -16384 as -infinity is
 * exact inside fits_i16 (simd/mod.rs:59-69).
 */
#include "esg_oracle.h"

#include <immintrin.h>
#include <stdlib.h>
#include <string.h>

#define W 32
#define NEG16 ((int16_t)-16384)
#define TRANSPOSED_MIN_READ_LEN 256

typedef struct eo_group {
    size_t len;          /* longest reference in the group: columns walked */
    int16_t lens[W];     /* per-lane reference length (0 for an empty lane) */
    int32_t refs[W];     /* per-lane panel index (-1 for an empty lane)     */
    int16_t* prof;       /* prof[(j * 5 + c) * W + lane]                    */
    int16_t* tprof;      /* tprof[(c * len + j) * W + lane], NEG16 past end */
    uint32_t* ends;      /* ends[j]: lanes whose last column is j           */
} eo_group;

struct eo_profile {
    uint32_t n_refs;
    size_t max_len;
    int32_t ma, mi, o, e;
    uint32_t n_groups;
    eo_group* groups;
    /* kept for the scalar fallback outside fits_i16 */
    const uint8_t** ref_ptr;
    uint32_t* ref_len;
    uint8_t* ref_store;
};

int eo_cpu_has_avx512bw(void)
{
    __builtin_cpu_init();
    return __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw");
}

static int16_t subst16(uint8_t c, uint8_t r, int32_t ma, int32_t mi)
{
    return (int16_t)((c == r || c == EO_WILDCARD || r == EO_WILDCARD) ? ma : mi);
}

typedef struct { uint32_t idx, len; } ref_key;

static int cmp_longest_first(const void* a, const void* b)
{
    const ref_key* x = (const ref_key*)a;
    const ref_key* y = (const ref_key*)b;
    if (x->len != y->len) return x->len > y->len ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);  /* stable */
}

eo_profile* eo_profile_build(const uint8_t* ref_codes, const uint64_t* ref_off,
                             const uint32_t* ref_len, uint32_t n_refs,
                             int32_t ma, int32_t mi, int32_t o, int32_t e)
{
    eo_profile* p = (eo_profile*)calloc(1, sizeof(eo_profile));
    p->n_refs = n_refs;
    p->ma = ma; p->mi = mi; p->o = o; p->e = e;
    size_t total = 0;
    for (uint32_t r = 0; r < n_refs; r++) {
        total += ref_len[r];
        if (ref_len[r] > p->max_len) p->max_len = ref_len[r];
    }
    p->ref_store = (uint8_t*)malloc(total ? total : 1);
    p->ref_ptr = (const uint8_t**)malloc(n_refs * sizeof(uint8_t*));
    p->ref_len = (uint32_t*)malloc(n_refs * sizeof(uint32_t));
    size_t at = 0;
    for (uint32_t r = 0; r < n_refs; r++) {
        memcpy(p->ref_store + at, ref_codes + ref_off[r], ref_len[r]);
        p->ref_ptr[r] = p->ref_store + at;
        p->ref_len[r] = ref_len[r];
        at += ref_len[r];
    }
    /* simd/mod.rs:294-296: longest first, stable. */
    ref_key* order = (ref_key*)malloc(n_refs * sizeof(ref_key));
    for (uint32_t r = 0; r < n_refs; r++) { order[r].idx = r; order[r].len = ref_len[r]; }
    qsort(order, n_refs, sizeof(ref_key), cmp_longest_first);
    p->n_groups = (n_refs + W - 1) / W;
    p->groups = (eo_group*)calloc(p->n_groups, sizeof(eo_group));
    for (uint32_t g = 0; g < p->n_groups; g++) {
        eo_group* G = &p->groups[g];
        const uint32_t first = g * W;
        const uint32_t cnt = (n_refs - first < W) ? n_refs - first : W;
        size_t len = 0;
        for (uint32_t k = 0; k < cnt; k++)
            if (order[first + k].len > len) len = order[first + k].len;
        G->len = len;
        const size_t lcols = len ? len : 1;
        G->prof = (int16_t*)aligned_alloc(64, ((lcols * EO_N_CODES * W * 2) + 63) / 64 * 64);
        G->tprof = (int16_t*)aligned_alloc(64, ((lcols * EO_N_CODES * W * 2) + 63) / 64 * 64);
        G->ends = (uint32_t*)calloc(lcols, sizeof(uint32_t));
        /* Padding scores as a mismatch in prof (masked out, simd/mod.rs:303). */
        for (size_t k = 0; k < len * EO_N_CODES * W; k++) G->prof[k] = (int16_t)mi;
        for (size_t k = 0; k < len * EO_N_CODES * W; k++) G->tprof[k] = NEG16;
        for (int lane = 0; lane < W; lane++) { G->lens[lane] = 0; G->refs[lane] = -1; }
        for (uint32_t lane = 0; lane < cnt; lane++) {
            const uint32_t ri = order[first + lane].idx;
            const uint8_t* codes = ref_codes + ref_off[ri];
            const uint32_t m = ref_len[ri];
            G->lens[lane] = (int16_t)m;
            G->refs[lane] = (int32_t)ri;
            if (m > 0) G->ends[m - 1] |= 1u << lane;
            for (uint32_t j = 0; j < m; j++)
                for (int c = 0; c < EO_N_CODES; c++) {
                    const int16_t s = subst16((uint8_t)c, codes[j], ma, mi);
                    G->prof[(j * EO_N_CODES + c) * W + lane] = s;
                    G->tprof[((size_t)c * len + j) * W + lane] = s;
                }
        }
    }
    free(order);
    return p;
}

void eo_profile_free(eo_profile* p)
{
    if (!p) return;
    for (uint32_t g = 0; g < p->n_groups; g++) {
        free(p->groups[g].prof);
        free(p->groups[g].tprof);
        free(p->groups[g].ends);
    }
    free(p->groups);
    free(p->ref_ptr);
    free(p->ref_len);
    free(p->ref_store);
    free(p);
}

/* avx512.rs:43-107 -- reference column j outer, read row i inner; per-row H/E
 * state (n * 32 lanes); masked column best. */
__attribute__((target("avx512f,avx512bw")))
static void kernel_row_major(const uint8_t* q, size_t n, const eo_group* g, int16_t o, int16_t e,
                             int local, int16_t* hbuf, int16_t* ebuf, int16_t* best)
{
    const __m512i zero = _mm512_setzero_si512();
    const __m512i neg = _mm512_set1_epi16(NEG16);
    const __m512i vo = _mm512_set1_epi16(o);
    const __m512i ve = _mm512_set1_epi16(e);
    __m512i* hp = (__m512i*)hbuf;
    __m512i* ep = (__m512i*)ebuf;
    for (size_t i = 0; i < n; i++) {
        _mm512_storeu_si512(hp + i, zero);
        _mm512_storeu_si512(ep + i, neg);
    }
    const __m512i lens = _mm512_loadu_si512((const void*)g->lens);
    __m512i acc = local ? zero : neg;
    for (size_t j = 0; j < g->len; j++) {
        const int16_t* pj = g->prof + j * EO_N_CODES * W;
        __m512i hdiag = zero, hup = zero, f = neg, colmax = neg;
        for (size_t i = 0; i < n; i++) {
            const __m512i s = _mm512_loadu_si512((const void*)(pj + (size_t)q[i] * W));
            const __m512i hleft = _mm512_loadu_si512(hp + i);
            const __m512i ev = _mm512_max_epi16(_mm512_add_epi16(hleft, vo),
                                                _mm512_add_epi16(_mm512_loadu_si512(ep + i), ve));
            _mm512_storeu_si512(ep + i, ev);
            __m512i h = _mm512_max_epi16(_mm512_add_epi16(hdiag, s), ev);
            hdiag = hleft;
            f = _mm512_max_epi16(_mm512_add_epi16(hup, vo), _mm512_add_epi16(f, ve));
            h = _mm512_max_epi16(h, f);
            if (local) h = _mm512_max_epi16(h, zero);
            _mm512_storeu_si512(hp + i, h);
            hup = h;
            colmax = _mm512_max_epi16(colmax, h);
        }
        const __mmask32 valid = _mm512_cmpgt_epi16_mask(lens, _mm512_set1_epi16((int16_t)j));
        if (local) {
            acc = _mm512_mask_max_epi16(acc, valid, acc, colmax);
        } else {
            acc = _mm512_mask_max_epi16(acc, valid, acc, hup);
            const __mmask32 last =
                _mm512_cmpeq_epi16_mask(lens, _mm512_set1_epi16((int16_t)(j + 1)));
            acc = _mm512_mask_max_epi16(acc, last, acc, colmax);
        }
    }
    _mm512_storeu_si512((void*)best, acc);
}

/* avx512.rs:278-354 -- read row outer, reference column inner; per-column
 * H/F state (len * 32 lanes); padding columns score NEG16 (tprof) so local
 * mode needs no mask; semi-global takes each lane's own last column inside
 * the row loop (ends) and the last row in one masked pass. */
__attribute__((target("avx512f,avx512bw")))
static void kernel_transposed(const uint8_t* q, size_t n, const eo_group* g, int16_t o, int16_t e,
                              int local, int16_t* hbuf, int16_t* fbuf, int16_t* best)
{
    const size_t l = g->len;
    const __m512i zero = _mm512_setzero_si512();
    const __m512i neg = _mm512_set1_epi16(NEG16);
    const __m512i vo = _mm512_set1_epi16(o);
    const __m512i ve = _mm512_set1_epi16(e);
    __m512i* hp = (__m512i*)hbuf;
    __m512i* fp = (__m512i*)fbuf;
    for (size_t j = 0; j < l; j++) {
        _mm512_storeu_si512(hp + j, zero);
        _mm512_storeu_si512(fp + j, neg);
    }
    __m512i acc = local ? zero : neg;
    for (size_t i = 0; i < n; i++) {
        const int16_t* row = g->tprof + (size_t)q[i] * l * W;
        __m512i hdiag = zero, hleft = zero, ev = neg;
        for (size_t j = 0; j < l; j++) {
            const __m512i s = _mm512_loadu_si512((const void*)(row + j * W));
            const __m512i hup = _mm512_loadu_si512(hp + j);
            const __m512i f = _mm512_max_epi16(_mm512_add_epi16(hup, vo),
                                               _mm512_add_epi16(_mm512_loadu_si512(fp + j), ve));
            _mm512_storeu_si512(fp + j, f);
            ev = _mm512_max_epi16(_mm512_add_epi16(hleft, vo), _mm512_add_epi16(ev, ve));
            __m512i h = _mm512_max_epi16(_mm512_add_epi16(hdiag, s), ev);
            hdiag = hup;
            h = _mm512_max_epi16(h, f);
            if (local) h = _mm512_max_epi16(h, zero);
            _mm512_storeu_si512(hp + j, h);
            hleft = h;
            if (local) {
                acc = _mm512_max_epi16(acc, h);
            } else {
                const uint32_t end = g->ends[j];
                if (end) acc = _mm512_mask_max_epi16(acc, (__mmask32)end, acc, h);
            }
        }
    }
    if (!local && n > 0) {
        const __m512i lens = _mm512_loadu_si512((const void*)g->lens);
        for (size_t j = 0; j < l; j++) {
            const __mmask32 valid = _mm512_cmpgt_epi16_mask(lens, _mm512_set1_epi16((int16_t)j));
            acc = _mm512_mask_max_epi16(acc, valid, acc, _mm512_loadu_si512(hp + j));
        }
    }
    _mm512_storeu_si512((void*)best, acc);
}

typedef struct { int16_t* h; int16_t* e; size_t cap; } scratch;

static void scratch_need(scratch* s, size_t elems)
{
    if (s->cap >= elems) return;
    free(s->h);
    free(s->e);
    s->h = (int16_t*)aligned_alloc(64, (elems * 2 + 63) / 64 * 64);
    s->e = (int16_t*)aligned_alloc(64, (elems * 2 + 63) / 64 * 64);
    s->cap = elems;
}

static void score_all_scratch(const eo_profile* p, const uint8_t* q, size_t n, int local,
                              int kernel, int32_t* out, scratch* sc)
{
    for (uint32_t r = 0; r < p->n_refs; r++) out[r] = 0;
    if (n == 0) return;
    /* mapper.rs:216-222: SIMD inside fits_i16, else the scalar oracle. */
    if (!eo_fits_i16(n, p->max_len, p->ma, p->mi, p->o, p->e)) {
        for (uint32_t r = 0; r < p->n_refs; r++)
            out[r] = eo_score(q, n, p->ref_ptr[r], p->ref_len[r], p->ma, p->mi, p->o, p->e, local);
        return;
    }
    const int transposed = kernel == 2 || (kernel == 0 && n >= TRANSPOSED_MIN_READ_LEN);
    int16_t best[W] __attribute__((aligned(64)));
    for (uint32_t g = 0; g < p->n_groups; g++) {
        const eo_group* G = &p->groups[g];
        if (transposed) {
            scratch_need(sc, (G->len ? G->len : 1) * W);
            kernel_transposed(q, n, G, (int16_t)p->o, (int16_t)p->e, local, sc->h, sc->e, best);
        } else {
            scratch_need(sc, n * W);
            kernel_row_major(q, n, G, (int16_t)p->o, (int16_t)p->e, local, sc->h, sc->e, best);
        }
        for (int lane = 0; lane < W; lane++)
            if (G->refs[lane] >= 0) out[G->refs[lane]] = best[lane];
    }
}

void eo_profile_score_all(const eo_profile* p, const uint8_t* q, size_t n, int local,
                          int kernel, int32_t* out)
{
    scratch sc = {0};
    score_all_scratch(p, q, n, local, kernel, out, &sc);
    free(sc.h);
    free(sc.e);
}

/* Reads per work unit handed to a worker: 64 as the reference's CLI
 * (align.rs:1470-1473); a bounded sample of very long reads needs smaller
 * units to keep every core busy. */
static int g_chunk = 64;

void eo_cpu_set_chunk(int reads) { g_chunk = reads > 0 ? reads : 64; }

int eo_cpu_map_batch(const eo_profile* p, const uint8_t* codes, const uint64_t* off,
                     const uint32_t* len, uint32_t n_reads, int both_strands, int local,
                     int threads, uint32_t cap, eo_result* results, uint32_t* ties,
                     int32_t* rows)
{
    int nt = threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    if (nt <= 0) nt = omp_get_max_threads();
#else
    if (nt <= 0) nt = 1;
#endif
    const uint32_t n_refs = p->n_refs;
#pragma omp parallel num_threads(nt)
    {
        scratch sc = {0};
        int32_t* fwd = (int32_t*)malloc((size_t)n_refs * sizeof(int32_t));
        int32_t* rev = (int32_t*)malloc((size_t)n_refs * sizeof(int32_t));
        uint8_t* rc = NULL;
        size_t rc_cap = 0;
#pragma omp for schedule(dynamic, g_chunk)
        for (long k = 0; k < (long)n_reads; k++) {
            const uint8_t* q = codes + off[k];
            const size_t n = len[k];
            eo_result* res = &results[k];
            if (n == 0) {
                res->best = EO_NO_SCORE;
                res->suboptimal = EO_NO_SCORE;
                res->n_tied = 0;
                res->flags = EO_RESULT_EMPTY;
                if (rows) {
                    memset(rows + (size_t)k * n_refs, 0, (size_t)n_refs * sizeof(int32_t));
                    if (both_strands)
                        memset(rows + ((size_t)n_reads + k) * n_refs, 0,
                               (size_t)n_refs * sizeof(int32_t));
                }
                continue;
            }
            score_all_scratch(p, q, n, local, 0, fwd, &sc);
            if (both_strands) {
                if (rc_cap < n) {
                    free(rc);
                    rc = (uint8_t*)malloc(n);
                    rc_cap = n;
                }
                eo_revcomp_codes(q, n, rc);
                score_all_scratch(p, rc, n, local, 0, rev, &sc);
            }
            eo_select(fwd, both_strands ? rev : NULL, n_refs, cap, res, ties + (size_t)k * cap);
            if (rows) {
                memcpy(rows + (size_t)k * n_refs, fwd, (size_t)n_refs * sizeof(int32_t));
                if (both_strands)
                    memcpy(rows + ((size_t)n_reads + k) * n_refs, rev,
                           (size_t)n_refs * sizeof(int32_t));
            }
        }
        free(fwd);
        free(rev);
        free(rc);
        free(sc.h);
        free(sc.e);
    }
    return nt;
}

/* The reference's CPU path for pairs, the timed baseline of the paired
 * workload: per pair (OpenMP, chunks of 32 pairs) pair_adapters
 * (align.rs:934-949), then the four mate rows with the SIMD kernels
 * (score_all, mapper.rs:242-252), the pair ranking (pair.rs:195-234) and
 * each mate's own both-strand selection (mapper.rs:444-472, the Separate
 * fallback).  mate_results / mate_ties may be NULL. */
int eo_cpu_map_pairs(const eo_profile* p, const uint8_t* codes, const uint64_t* off,
                     const uint32_t* len, uint32_t n_pairs, const uint8_t* a1, size_t al1,
                     const uint8_t* a2, size_t al2, size_t min_overlap, size_t max_read_len,
                     int both_strands, int local, int32_t min_score, int threads, uint32_t cap,
                     eo_pair_result* results, uint32_t* ties, eo_result* mate_results,
                     uint32_t* mate_ties, uint32_t* adapters)
{
    int nt = threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    if (nt <= 0) nt = omp_get_max_threads();
#else
    if (nt <= 0) nt = 1;
#endif
    const uint32_t n_refs = p->n_refs;
#pragma omp parallel num_threads(nt)
    {
        scratch sc = {0};
        int32_t* rows = (int32_t*)malloc((size_t)4 * n_refs * sizeof(int32_t));
        uint8_t* rc = NULL;
        size_t rc_cap = 0;
#pragma omp for schedule(dynamic, 32)
        for (long pp = 0; pp < (long)n_pairs; pp++) {
            const size_t a = 2 * (size_t)pp, b = a + 1;
            size_t ad[2] = {0, 0}, n[2];
            eo_pair_adapters(codes + off[a], len[a], codes + off[b], len[b], a1, al1, a2, al2,
                             min_overlap, max_read_len, ad);
            for (int m = 0; m < 2; m++) {
                const size_t l = len[a + m];
                n[m] = (max_read_len && l > max_read_len) ? 0 : l - ad[m];
                if (adapters) adapters[a + m] = (uint32_t)ad[m];
            }
            /* rows: mate m forward at 2m, reverse complement at 2m + 1 */
            for (int m = 0; m < 2; m++) {
                int32_t* f = rows + (size_t)(2 * m) * n_refs;
                int32_t* r = f + n_refs;
                if (n[m] == 0) {
                    memset(f, 0, (size_t)2 * n_refs * sizeof(int32_t));
                    continue;
                }
                const uint8_t* q = codes + off[a + m];
                if (rc_cap < n[m]) {
                    free(rc);
                    rc = (uint8_t*)malloc(n[m]);
                    rc_cap = n[m];
                }
                eo_revcomp_codes(q, n[m], rc);
                score_all_scratch(p, q, n[m], local, 0, f, &sc);
                score_all_scratch(p, rc, n[m], local, 0, r, &sc);
            }
            eo_pair_result* res = &results[pp];
            if (n[0] == 0 || n[1] == 0) {
                res->best = res->next = EO_NO_SCORE;
                res->n_tied = 0;
                res->flags = EO_RESULT_EMPTY;
                res->xs[0] = res->xs[1] = res->primary[0] = res->primary[1] = EO_NO_SCORE;
            } else {
                eo_pair_select(rows, rows + n_refs, rows + 2 * (size_t)n_refs,
                               rows + 3 * (size_t)n_refs, n_refs, both_strands, min_score, cap,
                               res, ties + (size_t)pp * cap);
            }
            if (mate_results)
                for (int m = 0; m < 2; m++) {
                    eo_result* mr = &mate_results[a + m];
                    if (n[m] == 0) {
                        mr->best = mr->suboptimal = EO_NO_SCORE;
                        mr->n_tied = 0;
                        mr->flags = EO_RESULT_EMPTY;
                        continue;
                    }
                    eo_select(rows + (size_t)(2 * m) * n_refs, rows + (size_t)(2 * m + 1) * n_refs,
                              n_refs, cap, mr, mate_ties + (a + m) * cap);
                }
        }
        free(rows);
        free(rc);
        free(sc.h);
        free(sc.e);
    }
    return nt;
}
