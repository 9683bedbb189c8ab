/*
 * esg_pairs.c -- restatement of eschalign's paired-end scoring inputs and
 * candidate ranking.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see esg_oracle.h).
 *   - eo_adapter_find         crates/eschalign/src/adapter.rs:68-91
 *   - eo_adapter_detect_pair  crates/eschalign/src/adapter.rs:95-110
 *   - eo_pair_adapters        crates/eschalign-cli/src/align.rs:934-949
 *   - eo_pair_select          crates/eschalign/src/mapper/pair.rs:195-234 (candidates,
 *                             eligibility, order; the first tier and the next one)
 *                             and :297-314 (per-mate XS outside the tie set)
 */
#include "esg_oracle.h"

#include <stdlib.h>
#include <string.h>

/* adapter.rs:68-91.  Codes in, wildcards match; the leftmost position whose
 * overlap (the adapter's prefix against the read's rest) has at most one
 * mismatch per ten bases; everything from there is adapter. */
size_t eo_adapter_find(const uint8_t* read, size_t n, const uint8_t* adapter, size_t a,
                       size_t min_overlap)
{
    if (min_overlap < 1) min_overlap = 1;
    if (n < min_overlap || a == 0) return 0;
    for (size_t p = 0; p + min_overlap <= n; p++) {
        const size_t overlap = a < n - p ? a : n - p;
        if (overlap < min_overlap) break;
        size_t mism = 0;
        for (size_t k = 0; k < overlap; k++) {
            const uint8_t x = read[p + k], y = adapter[k];
            if (x != y && x != EO_WILDCARD && y != EO_WILDCARD) mism++;
        }
        if (mism <= overlap / 10) return n - p;
    }
    return 0;
}

/* adapter.rs:95-110: both mates searched; where they disagree about the
 * insert end, the weaker detection (shorter overlap) is dropped, both on a
 * tie. */
void eo_adapter_detect_pair(const uint8_t* r1, size_t l1, const uint8_t* r2, size_t l2,
                            const uint8_t* a1, size_t al1, const uint8_t* a2, size_t al2,
                            size_t min_overlap, size_t out[2])
{
    size_t ad0 = eo_adapter_find(r1, l1, a1, al1, min_overlap);
    size_t ad1 = eo_adapter_find(r2, l2, a2, al2, min_overlap);
    if (ad0 > 0 && ad1 > 0 && l1 - ad0 != l2 - ad1) {
        const size_t e1 = ad0 < al1 ? ad0 : al1, e2 = ad1 < al2 ? ad1 : al2;
        if (e1 > e2) ad1 = 0;
        else if (e1 < e2) ad0 = 0;
        else ad0 = ad1 = 0;
    }
    out[0] = ad0;
    out[1] = ad1;
}

/* crates/eschalign-cli/src/align.rs:934-949 (pair_adapters): a mate longer
 * than max_read_len (0 = no limit) is not aligned and not searched; the
 * other mate is then searched alone. */
void eo_pair_adapters(const uint8_t* r1, size_t l1, const uint8_t* r2, size_t l2,
                      const uint8_t* a1, size_t al1, const uint8_t* a2, size_t al2,
                      size_t min_overlap, size_t max_read_len, size_t out[2])
{
    const int o1 = max_read_len && l1 > max_read_len, o2 = max_read_len && l2 > max_read_len;
    out[0] = out[1] = 0;
    if (!o1 && !o2)
        eo_adapter_detect_pair(r1, l1, r2, l2, a1, al1, a2, al2, min_overlap, out);
    else if (!o1)
        out[0] = eo_adapter_find(r1, l1, a1, al1, min_overlap);
    else if (!o2)
        out[1] = eo_adapter_find(r2, l2, a2, al2, min_overlap);
}

/* pair.rs:195-234 and :297-314.  Candidate (reference r, template strand t):
 * mate 1 as sequenced and mate 2 reverse-complemented on t = 0, the reverse
 * on t = 1 (mate_reverse, pair.rs:135-137); eligible when both mates score
 * at least min_score; sum = both scores.  Candidates in order (-sum, r, t):
 * the best sum, how many candidates share it (the first tier), the first
 * `cap` of them as (r << 1) | t, the next tier's sum, the primary's two mate
 * scores, and per mate the best score over every candidate outside the first
 * tier (the XS of a pair whose whole first tier passes the pair
 * constraints).  A pair with an empty mate has no candidates
 * (pair.rs:182-184). */
void eo_pair_select(const int32_t* f0, const int32_t* r0, const int32_t* f1, const int32_t* r1,
                    uint32_t n_refs, int both_strands, int32_t min_score, uint32_t cap,
                    eo_pair_result* out, uint32_t* ties)
{
    int32_t best = EO_NO_SCORE, next = EO_NO_SCORE;
    int any = 0;
    const int nt = both_strands ? 2 : 1;
    for (uint32_t r = 0; r < n_refs; r++)
        for (int t = 0; t < nt; t++) {
            const int32_t a = t ? r0[r] : f0[r], b = t ? f1[r] : r1[r];
            if (a < min_score || b < min_score) continue;
            if (!any || a + b > best) best = a + b;
            any = 1;
        }
    uint32_t n = 0;
    int32_t xs[2] = {EO_NO_SCORE, EO_NO_SCORE}, prim[2] = {EO_NO_SCORE, EO_NO_SCORE};
    for (uint32_t r = 0; r < n_refs; r++)
        for (int t = 0; t < nt; t++) {
            const int32_t a = t ? r0[r] : f0[r], b = t ? f1[r] : r1[r];
            const int elig = a >= min_score && b >= min_score;
            if (elig && a + b == best) {
                if (n == 0) {
                    prim[0] = a;
                    prim[1] = b;
                }
                if (n < cap) ties[n] = (r << 1) | (uint32_t)t;
                n++;
                continue;
            }
            if (elig && a + b > next) next = a + b;
            if (a > xs[0]) xs[0] = a;
            if (b > xs[1]) xs[1] = b;
        }
    out->best = best;
    out->next = next;
    out->n_tied = n;
    out->flags = (any ? 0 : EO_RESULT_EMPTY) | (n > cap ? EO_RESULT_TIES_TRUNCATED : 0);
    out->xs[0] = xs[0];
    out->xs[1] = xs[1];
    out->primary[0] = prim[0];
    out->primary[1] = prim[1];
}

/* Pairs end to end with the scalar oracle: mate codes 2 per pair (mate 1,
 * mate 2), already trimmed; rows of the four queries per pair, then the
 * selection.  A pair with an empty mate has no candidates (pair.rs:182-184). */
int eo_scalar_map_pairs(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                        uint32_t n_pairs, const uint8_t* ref_codes, const uint64_t* ref_off,
                        const uint32_t* ref_len, uint32_t n_refs, int32_t ma, int32_t mi,
                        int32_t o, int32_t e, int both_strands, int local, int32_t min_score,
                        int threads, uint32_t cap, eo_pair_result* results, uint32_t* ties)
{
    int nt = threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    if (nt <= 0) nt = omp_get_max_threads();
#else
    if (nt <= 0) nt = 1;
#endif
#pragma omp parallel num_threads(nt)
    {
        int32_t* rows = (int32_t*)malloc((size_t)4 * n_refs * sizeof(int32_t));
        uint8_t* rc = NULL;
        size_t rc_cap = 0;
#pragma omp for schedule(dynamic, 32)
        for (long p = 0; p < (long)n_pairs; p++) {
            eo_pair_result* res = &results[p];
            const uint32_t n0 = len[2 * p], n1 = len[2 * p + 1];
            if (n0 == 0 || n1 == 0) {
                res->best = res->next = EO_NO_SCORE;
                res->n_tied = 0;
                res->flags = EO_RESULT_EMPTY;
                res->xs[0] = res->xs[1] = res->primary[0] = res->primary[1] = EO_NO_SCORE;
                continue;
            }
            for (int m = 0; m < 2; m++) {
                const uint8_t* q = codes + off[2 * p + m];
                const size_t n = len[2 * p + m];
                if (rc_cap < n) {
                    free(rc);
                    rc = (uint8_t*)malloc(n);
                    rc_cap = n;
                }
                eo_revcomp_codes(q, n, rc);
                for (uint32_t r = 0; r < n_refs; r++) {
                    rows[(2 * m) * n_refs + r] =
                        eo_score(q, n, ref_codes + ref_off[r], ref_len[r], ma, mi, o, e, local);
                    rows[(2 * m + 1) * n_refs + r] =
                        eo_score(rc, n, ref_codes + ref_off[r], ref_len[r], ma, mi, o, e, local);
                }
            }
            eo_pair_select(rows, rows + n_refs, rows + 2 * n_refs, rows + 3 * n_refs, n_refs,
                           both_strands, min_score, cap, res, ties + (size_t)p * cap);
        }
        free(rows);
        free(rc);
    }
    return nt;
}

/* The ranking alone over rows laid out as the CUDA path lays them out:
 * forward rows of the 2 n_pairs mates, then their reverse-complement rows.
 * Mate lengths decide emptiness (pair.rs:182-184). */
void eo_pairs_from_rows(const int32_t* rows, const uint32_t* len, uint32_t n_pairs,
                        uint32_t n_refs, int both_strands, int32_t min_score, uint32_t cap,
                        eo_pair_result* results, uint32_t* ties)
{
    const size_t nr = n_refs, n_reads = 2 * (size_t)n_pairs;
    for (size_t p = 0; p < n_pairs; p++) {
        eo_pair_result* res = &results[p];
        if (len[2 * p] == 0 || len[2 * p + 1] == 0) {
            res->best = res->next = EO_NO_SCORE;
            res->n_tied = 0;
            res->flags = EO_RESULT_EMPTY;
            res->xs[0] = res->xs[1] = res->primary[0] = res->primary[1] = EO_NO_SCORE;
            continue;
        }
        const int32_t* f0 = rows + (2 * p) * nr;
        const int32_t* r0 = rows + (n_reads + 2 * p) * nr;
        eo_pair_select(f0, r0, f0 + nr, r0 + nr, n_refs, both_strands, min_score, cap, res,
                       ties + p * cap);
    }
}
