/*
 * esg_oracle.c -- scalar restatement of eschalign's panel-scoring semantics.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see esg_oracle.h).  Each function
 * cites the reference file:line it restates.  Integer arithmetic throughout,
 * compared by equality, as the reference's own tests do
 * (crates/eschalign/src/scalar.rs:5-7).
 */
#include "esg_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

/* scalar.rs:42 -- stand-in for -infinity that survives adding a penalty. */
#define EO_NEG (INT32_MIN / 4)

/* alphabet.rs:29-50 */
uint8_t eo_encode_base(uint8_t b)
{
    switch (b) {
    case 'A': case 'a': return EO_A;
    case 'C': case 'c': return EO_C;
    case 'G': case 'g': return EO_G;
    case 'T': case 't': case 'U': case 'u': return EO_T;
    default: return EO_WILDCARD;
    }
}

void eo_encode(const uint8_t* letters, size_t n, uint8_t* codes)
{
    for (size_t i = 0; i < n; i++) codes[i] = eo_encode_base(letters[i]);
}

/* alphabet.rs:58-64 */
void eo_revcomp_codes(const uint8_t* codes, size_t n, uint8_t* out)
{
    for (size_t i = 0; i < n; i++) {
        uint8_t c = codes[n - 1 - i];
        out[i] = (c == EO_WILDCARD) ? EO_WILDCARD : (uint8_t)(3 - c);
    }
}

/* scoring.rs:70-100 (MAX_SCORE_MAGNITUDE = 1000, scoring.rs:14) */
int eo_scoring_validate(int32_t ma, int32_t mi, int32_t o, int32_t e)
{
    if (ma <= 0) return 1;
    if (mi >= ma) return 2;
    if (o > 0 || e > 0) return 3;
    const int32_t v[4] = {ma, mi, o, e};
    for (int k = 0; k < 4; k++)
        if (abs(v[k]) > 1000) return 4;
    return 0;
}

/* scoring.rs:105-111: a match if equal or either is the wildcard. */
static inline int32_t subst(uint8_t a, uint8_t b, int32_t ma, int32_t mi)
{
    return (a == b || a == EO_WILDCARD || b == EO_WILDCARD) ? ma : mi;
}

static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

/* scalar.rs:120-163.  Column j outer over the reference, row i inner over
 * the read; zero border, E/F = -inf on it; local floors at zero and takes
 * the best cell anywhere; semi-global takes the best of the last row (every
 * column) and of the last column (every row). */
int32_t eo_score(const uint8_t* q, size_t n, const uint8_t* r, size_t m,
                 int32_t ma, int32_t mi, int32_t o, int32_t e, int local)
{
    if (n == 0 || m == 0) return 0;
    int32_t* hcol = (int32_t*)malloc((n + 1) * sizeof(int32_t));
    int32_t* ecol = (int32_t*)malloc((n + 1) * sizeof(int32_t));
    for (size_t i = 0; i <= n; i++) { hcol[i] = 0; ecol[i] = EO_NEG; }
    int32_t best = local ? 0 : EO_NEG;
    for (size_t j = 0; j < m; j++) {
        const uint8_t rj = r[j];
        int32_t hdiag = 0, hup = 0, f = EO_NEG, colmax = EO_NEG;
        for (size_t i = 1; i <= n; i++) {
            const int32_t hleft = hcol[i];
            const int32_t ev = imax(hleft + o, ecol[i] + e);
            ecol[i] = ev;
            f = imax(hup + o, f + e);
            int32_t h = imax(imax(hdiag + subst(q[i - 1], rj, ma, mi), ev), f);
            if (local) h = imax(h, 0);
            hdiag = hleft;
            hcol[i] = h;
            hup = h;
            colmax = imax(colmax, h);
        }
        if (local) {
            best = imax(best, colmax);
        } else {
            best = imax(best, hup);
            if (j + 1 == m) best = imax(best, colmax);
        }
    }
    free(hcol);
    free(ecol);
    return best;
}

/* simd/mod.rs:222-227 */
int eo_fits_i16(size_t n, size_t max_ref_len, int32_t ma, int32_t mi, int32_t o, int32_t e)
{
    const int64_t k = (int64_t)(n < max_ref_len ? n : max_ref_len);
    const int64_t mm = imax(abs(ma), abs(mi));
    const int64_t bound = k * mm + abs(o) + abs(e);
    return bound < 15000 && max_ref_len < 15000;
}

/* mapper.rs:444-472.  Candidate order: reference order, forward before
 * reverse.  best = max; the tie set = every candidate equal to best, counted
 * in full; suboptimal = max over candidates not equal to best (none when all
 * tie). */
void eo_select(const int32_t* fwd, const int32_t* rev, uint32_t n_refs, uint32_t cap,
               eo_result* out, uint32_t* ties)
{
    int32_t best = INT32_MIN;
    for (uint32_t r = 0; r < n_refs; r++) {
        best = imax(best, fwd[r]);
        if (rev) best = imax(best, rev[r]);
    }
    uint32_t n_tied = 0;
    int32_t sub = EO_NO_SCORE;
    int have_sub = 0;
    for (uint32_t r = 0; r < n_refs; r++) {
        for (int s = 0; s < (rev ? 2 : 1); s++) {
            const int32_t v = s ? rev[r] : fwd[r];
            if (v == best) {
                if (n_tied < cap) ties[n_tied] = (r << 1) | (uint32_t)s;
                n_tied++;
            } else if (!have_sub || v > sub) {
                sub = v;
                have_sub = 1;
            }
        }
    }
    out->best = best;
    out->suboptimal = have_sub ? sub : EO_NO_SCORE;
    out->n_tied = n_tied;
    out->flags = n_tied > cap ? EO_RESULT_TIES_TRUNCATED : 0;
}

static int eo_threads(int threads)
{
    if (threads > 0) return threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void eo_score_matrix(const uint8_t* codes, const uint64_t* off, const uint32_t* len, uint32_t n_q,
                     const uint8_t* ref_codes, const uint64_t* ref_off, const uint32_t* ref_len,
                     uint32_t n_refs, int32_t ma, int32_t mi, int32_t o, int32_t e, int local,
                     int threads, int32_t* out)
{
    const int nt = eo_threads(threads);
    (void)nt;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nt)
    for (long k = 0; k < (long)n_q; k++) {
        for (uint32_t r = 0; r < n_refs; r++)
            out[(size_t)k * n_refs + r] = eo_score(codes + off[k], len[k], ref_codes + ref_off[r],
                                                   ref_len[r], ma, mi, o, e, local);
    }
}

int eo_scalar_map_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                        uint32_t n_reads, const uint8_t* ref_codes, const uint64_t* ref_off,
                        const uint32_t* ref_len, uint32_t n_refs, int32_t ma, int32_t mi,
                        int32_t o, int32_t e, int both_strands, int local, int threads,
                        uint32_t cap, eo_result* results, uint32_t* ties, int32_t* rows)
{
    const int nt = eo_threads(threads);
#pragma omp parallel num_threads(nt)
    {
        int32_t* fwd = (int32_t*)malloc((size_t)n_refs * sizeof(int32_t));
        int32_t* rev = (int32_t*)malloc((size_t)n_refs * sizeof(int32_t));
        uint8_t* rc = NULL;
        size_t rc_cap = 0;
#pragma omp for schedule(dynamic, 64)
        for (long k = 0; k < (long)n_reads; k++) {
            const uint8_t* q = codes + off[k];
            const size_t n = len[k];
            eo_result* res = &results[k];
            if (n == 0) {
                /* mapper.rs:417-426: an empty read has no candidates. */
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
            for (uint32_t r = 0; r < n_refs; r++)
                fwd[r] = eo_score(q, n, ref_codes + ref_off[r], ref_len[r], ma, mi, o, e, local);
            if (both_strands) {
                if (rc_cap < n) {
                    free(rc);
                    rc = (uint8_t*)malloc(n);
                    rc_cap = n;
                }
                eo_revcomp_codes(q, n, rc);
                for (uint32_t r = 0; r < n_refs; r++)
                    rev[r] = eo_score(rc, n, ref_codes + ref_off[r], ref_len[r], ma, mi, o, e,
                                      local);
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
    }
    return nt;
}
