/*
 * esg_align.c -- restatement of eschalign's traceback alignment.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see esg_oracle.h).
 *   - eo_align: crates/eschalign/src/scalar.rs:182-206 (align), :213-289
 *     (fill: the traceback DP, one trace code per cell, the end cell as the
 *     first maximum of a column-major scan) and :292-364 (walk: diagonal,
 *     then insertion, then deletion; extending inside a gap; local mode
 *     stops at the first zero cell).
 * Ops are written run-length encoded as BAM CIGAR words (len << 4 | op with
 * M = 0, I = 1, D = 2), first to last.
 */
#include "esg_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NEG (INT32_MIN / 4)
/* trace codes (scalar.rs:167-175) */
#define T_STOP 0
#define T_DIAG 1
#define T_INS 2
#define T_DEL 3
#define T_E_EXT 4
#define T_F_EXT 8

static int32_t sub_of(uint8_t a, uint8_t b, int32_t ma, int32_t mi)
{
    return (a == b || a == EO_WILDCARD || b == EO_WILDCARD) ? ma : mi;
}

int eo_align(const uint8_t* q, size_t n, const uint8_t* r, size_t m, int32_t ma, int32_t mi,
             int32_t o, int32_t e, int local, eo_alignment* out, uint32_t* ops, size_t ops_cap)
{
    memset(out, 0, sizeof *out);
    if (n == 0 || m == 0) return 0;
    const size_t rows = n + 1;
    uint8_t* trace = (uint8_t*)calloc(rows * (m + 1), 1);
    int32_t* hcol = (int32_t*)calloc(rows, sizeof(int32_t));
    int32_t* ecol = (int32_t*)malloc(rows * sizeof(int32_t));
    if (!trace || !hcol || !ecol) {
        free(trace);
        free(hcol);
        free(ecol);
        return -1;
    }
    for (size_t i = 0; i < rows; i++) ecol[i] = NEG;
    int32_t best = local ? 0 : NEG;
    size_t bi = 0, bj = 0;
    for (size_t j = 1; j <= m; j++) {
        const uint8_t rj = r[j - 1];
        uint8_t* col = trace + j * rows;
        int32_t hdiag = 0, hup = 0, f = NEG;
        const int last_col = j == m;
        for (size_t k = 0; k < n; k++) {
            const int32_t hleft = hcol[k + 1];
            const int32_t e_open = hleft + o, e_ext = ecol[k + 1] + e;
            const int32_t ev = e_open > e_ext ? e_open : e_ext;
            const int32_t f_open = hup + o, f_ext = f + e;
            f = f_open > f_ext ? f_open : f_ext;
            const int32_t hd = hdiag + sub_of(q[k], rj, ma, mi);
            int32_t h = hd > ev ? hd : ev;
            if (f > h) h = f;
            if (local && h < 0) h = 0;
            uint8_t t = h == f ? T_INS : T_DEL;
            if (h == hd) t = T_DIAG;
            if (local && h == 0) t = T_STOP;
            if (ev == e_ext) t |= T_E_EXT;
            if (f == f_ext) t |= T_F_EXT;
            col[k + 1] = t;
            ecol[k + 1] = ev;
            hdiag = hleft;
            hcol[k + 1] = h;
            hup = h;
            if ((local || last_col) && h > best) {
                best = h;
                bi = k + 1;
                bj = j;
            }
        }
        if (!local && !last_col && hup > best) {
            best = hup;
            bi = n;
            bj = j;
        }
    }
    /* walk */
    int rc = 0;
    if (bi && bj) {
        size_t i = bi, j = bj, n_rev = 0;
        uint8_t* rev = (uint8_t*)malloc(n + m + 1);
        int state = 0; /* 0 H, 1 E, 2 F */
        while (i > 0 && j > 0) {
            const uint8_t t = trace[j * rows + i];
            if (state == 0) {
                const uint8_t src = t & 3;
                if (src == T_STOP) break;
                if (src == T_DIAG) {
                    rev[n_rev++] = 0;
                    i--;
                    j--;
                } else if (src == T_INS) {
                    state = 2;
                } else {
                    state = 1;
                }
            } else if (state == 2) {
                rev[n_rev++] = 1;
                if (!(t & T_F_EXT)) state = 0;
                i--;
            } else {
                rev[n_rev++] = 2;
                if (!(t & T_E_EXT)) state = 0;
                j--;
            }
        }
        size_t w = 0;
        for (size_t k = n_rev; k-- > 0;) {
            const uint32_t op = rev[k];
            if (w && (ops[w - 1] & 0xf) == op) {
                ops[w - 1] += 16;
            } else if (w < ops_cap) {
                ops[w++] = 16 | op;
            } else {
                rc = -2;
                break;
            }
        }
        free(rev);
        out->score = best;
        out->query_start = (uint32_t)i;
        out->query_end = (uint32_t)bi;
        out->ref_start = (uint32_t)j;
        out->ref_end = (uint32_t)bj;
        out->n_ops = (uint32_t)w;
    }
    free(trace);
    free(hcol);
    free(ecol);
    return rc;
}

/* The reference's CPU traceback of a batch of winners, the timed baseline:
 * eo_align per job over OpenMP threads (the scalar path; the reference runs
 * the same walk over its SIMD trace_pairs for up to 32 jobs at a time).
 * Job k aligns read job_read[k] (reverse-complemented when job_rev[k])
 * against reference job_ref[k]; ops go to ops + k * ops_stride. */
int eo_align_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                   const uint8_t* ref_codes, const uint64_t* ref_off, const uint32_t* ref_len,
                   const uint32_t* job_read, const uint32_t* job_ref, const uint8_t* job_rev,
                   uint32_t n_jobs, int32_t ma, int32_t mi, int32_t o, int32_t e, int local,
                   int threads, eo_alignment* out, uint32_t* ops, size_t ops_stride)
{
    int nt = threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    if (nt <= 0) nt = omp_get_max_threads();
#else
    if (nt <= 0) nt = 1;
#endif
    int bad = 0;
#pragma omp parallel num_threads(nt)
    {
        uint8_t* rc = NULL;
        size_t rc_cap = 0;
#pragma omp for schedule(dynamic, 64)
        for (long k = 0; k < (long)n_jobs; k++) {
            const uint8_t* q = codes + off[job_read[k]];
            const size_t n = len[job_read[k]];
            if (job_rev[k]) {
                if (rc_cap < n) {
                    free(rc);
                    rc = (uint8_t*)malloc(n ? n : 1);
                    rc_cap = n;
                }
                eo_revcomp_codes(q, n, rc);
                q = rc;
            }
            if (eo_align(q, n, ref_codes + ref_off[job_ref[k]], ref_len[job_ref[k]], ma, mi, o,
                         e, local, &out[k], ops + (size_t)k * ops_stride, ops_stride))
                bad = 1;
        }
        free(rc);
    }
    return bad ? -1 : nt;
}

/* crates/eschalign/src/sam.rs:76-121 (md_nm) with calmd_match (sam.rs:63-69)
 * on codes. */
static int put_run(char* md, size_t cap, size_t* at, uint32_t run)
{
    char buf[16];
    const int w = snprintf(buf, sizeof buf, "%u", run);
    if (*at + (size_t)w > cap) return -1;
    memcpy(md + *at, buf, (size_t)w);
    *at += (size_t)w;
    return 0;
}

static char md_letter(const uint8_t* rc, const uint8_t* rl, size_t j)
{
    if (rl) {
        const uint8_t c = rl[j];
        return (char)((c >= 'a' && c <= 'z') ? c - 32 : c);
    }
    return "ACGTN"[rc[j] > 4 ? 4 : rc[j]];
}

long eo_md_nm(const uint8_t* q, size_t n, int reverse, const uint8_t* ref_codes,
              const uint8_t* ref_letters, const eo_alignment* a, const uint32_t* ops, char* md,
              size_t md_cap, uint32_t* nm_out)
{
    size_t at = 0, i = a->query_start, j = a->ref_start;
    uint32_t run = 0, nm = 0;
    for (uint32_t k = 0; k < a->n_ops; k++) {
        const uint32_t op = ops[k] & 0xfu, l = ops[k] >> 4;
        if (op == 0) {
            for (uint32_t t = 0; t < l; t++, i++, j++) {
                uint32_t x = reverse ? q[n - 1 - i] : q[i];
                x = x > 4 ? 4 : x;
                if (reverse && x < 4) x = 3 - x;
                const uint32_t y = ref_codes[j] > 4 ? 4 : ref_codes[j];
                if (x == y && y < 4) {
                    run++;
                } else {
                    if (put_run(md, md_cap, &at, run) || at + 1 > md_cap) return -1;
                    md[at++] = md_letter(ref_codes, ref_letters, j);
                    run = 0;
                    nm++;
                }
            }
        } else if (op == 1) {
            i += l;
            nm += l;
        } else {
            if (put_run(md, md_cap, &at, run) || at + 1 + l > md_cap) return -1;
            md[at++] = '^';
            for (uint32_t t = 0; t < l; t++) md[at++] = md_letter(ref_codes, ref_letters, j + t);
            run = 0;
            j += l;
            nm += l;
        }
    }
    if (put_run(md, md_cap, &at, run)) return -1;
    *nm_out = nm;
    return (long)at;
}

int eo_md_nm_batch(const uint8_t* codes, const uint64_t* off, const uint32_t* len,
                   const uint8_t* ref_codes, const uint64_t* ref_off, const uint8_t* ref_letters,
                   const uint32_t* job_read, const uint32_t* job_ref, const uint8_t* job_rev,
                   const eo_alignment* al, const uint32_t* ops, size_t ops_stride,
                   uint32_t n_jobs, int threads, char* md, size_t md_stride, uint32_t* md_len,
                   uint32_t* nm)
{
    int nt = threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    if (nt <= 0) nt = omp_get_max_threads();
#else
    if (nt <= 0) nt = 1;
#endif
    int bad = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256)
    for (long k = 0; k < (long)n_jobs; k++) {
        const uint64_t ro = ref_off[job_ref[k]];
        const long w = eo_md_nm(codes + off[job_read[k]], len[job_read[k]], job_rev[k],
                                ref_codes + ro, ref_letters ? ref_letters + ro : NULL, &al[k],
                                ops + (size_t)k * ops_stride, md + (size_t)k * md_stride,
                                md_stride, &nm[k]);
        if (w < 0) bad = 1;
        else md_len[k] = (uint32_t)w;
    }
    return bad ? -1 : nt;
}
