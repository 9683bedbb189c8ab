/* A consumer of the C ABI written in C, as a binding in another compiled
 * language would use it: plain pointers and sizes, no Python.  It runs the
 * host half of the CLI's unpaired BAM run with mappings computed elsewhere
 * (the mapping stage's arrays, handed over with esg_mapping_from_arrays):
 *
 *   unpaired_bam IN.bam OUT.bam HEADER.txt REFS.txt MAPPING.bin SECONDARY SORT MAX_READ_LEN
 *
 * REFS.txt: one "name length" line per panel reference.  MAPPING.bin: the
 * counts n_reads, n_hits, n_ops, n_md (u64 each), then the esg_read_mapping,
 * esg_hit, CIGAR-word and MD arrays of every read of IN.bam in input order.
 * Reads are taken seven at a time; each batch's records are encoded and the
 * chunks pushed to the writer out of order (1, 0, then the rest).  Exits 0
 * after printing "records N". */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "eschalign_b200.h"

static void die(const char* what, esg_status st) {
    fprintf(stderr, "%s: %s (%s)\n", what, esg_status_string(st), esg_last_error());
    exit(1);
}

static void* slurp(const char* path, size_t* n) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(1);
    }
    fseek(f, 0, SEEK_END);
    long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char* buf = malloc((size_t)len + 1);
    if (!buf || fread(buf, 1, (size_t)len, f) != (size_t)len) {
        fprintf(stderr, "reading %s failed\n", path);
        exit(1);
    }
    buf[len] = 0;
    fclose(f);
    *n = (size_t)len;
    return buf;
}

int main(int argc, char** argv) {
    if (argc != 9) {
        fprintf(stderr, "usage: %s IN OUT HEADER REFS MAPPING SECONDARY SORT MAX_READ_LEN\n",
                argv[0]);
        return 2;
    }
    if (esg_abi_version() != 1) {
        fprintf(stderr, "unexpected ABI version %d\n", esg_abi_version());
        return 1;
    }
    const uint32_t secondary = (uint32_t)atoi(argv[6]);
    const int32_t sort = atoi(argv[7]);
    const uint32_t max_read_len = (uint32_t)atoi(argv[8]);

    size_t n_header = 0, n_refs_text = 0, n_map = 0;
    char* header = slurp(argv[3], &n_header);
    char* refs_text = slurp(argv[4], &n_refs_text);
    char* names[256];
    uint32_t lens[256], n_refs = 0;
    for (char* line = strtok(refs_text, "\n"); line && n_refs < 256; line = strtok(NULL, "\n")) {
        char* sp = strchr(line, ' ');
        if (!sp) continue;
        *sp = 0;
        names[n_refs] = line;
        lens[n_refs++] = (uint32_t)strtoul(sp + 1, NULL, 10);
    }

    const uint8_t* map = slurp(argv[5], &n_map);
    uint64_t counts[4];
    memcpy(counts, map, sizeof counts);
    const esg_read_mapping* reads = (const esg_read_mapping*)(map + sizeof counts);
    const esg_hit* hits = (const esg_hit*)(reads + counts[0]);
    const uint32_t* ops = (const uint32_t*)(hits + counts[1]);
    const char* md = (const char*)(ops + counts[2]);
    if ((const uint8_t*)md + counts[3] != map + n_map) {
        fprintf(stderr, "mapping file size does not match its counts\n");
        return 1;
    }

    esg_bam_reader* rd = NULL;
    esg_status st = esg_bam_open(argv[1], 2, &rd);
    if (st != ESG_OK) die("esg_bam_open", st);
    esg_bam_writer* wr = NULL;
    st = esg_bam_writer_open(argv[2], header, (const char* const*)names, lens, n_refs, sort, 2,
                             &wr);
    if (st != ESG_OK) die("esg_bam_writer_open", st);

    esg_bam_records* held = NULL; /* chunk 0, pushed after chunk 1 */
    esg_bam_options opt = {secondary, 0};
    uint64_t at = 0, seq = 0, records = 0;
    for (;;) {
        esg_bam_batch* b = NULL;
        st = esg_bam_read_batch(rd, 7, max_read_len, &b);
        if (st != ESG_OK) die("esg_bam_read_batch", st);
        const uint8_t* codes;
        const uint64_t* off;
        const uint32_t* len;
        uint32_t n = 0;
        st = esg_bam_batch_reads(b, &codes, &off, &len, &n);
        if (st != ESG_OK) die("esg_bam_batch_reads", st);
        if (n == 0) {
            esg_bam_batch_free(b);
            break;
        }
        if (at + n > counts[0]) {
            fprintf(stderr, "the BAM holds more reads than the mapping\n");
            return 1;
        }
        /* this batch's reads; their hits, CIGAR words and MD stay in the
         * whole arrays, which their offsets index */
        esg_mapping* m = NULL;
        st = esg_mapping_from_arrays(reads + at, n, hits, counts[1], ops, counts[2], md,
                                     counts[3], &m);
        if (st != ESG_OK) die("esg_mapping_from_arrays", st);
        esg_bam_records* r = NULL;
        st = esg_bam_encode(b, m, &opt, (const char* const*)names, n_refs, 2, &r);
        if (st != ESG_OK) die("esg_bam_encode", st);
        uint64_t n_bytes = 0;
        uint32_t n_rec = 0;
        esg_bam_records_bytes(r, &n_bytes, &n_rec);
        records += n_rec;
        if (seq == 0) {
            held = r;
        } else {
            st = esg_bam_writer_push(wr, seq, r);
            if (st != ESG_OK) die("esg_bam_writer_push", st);
            esg_bam_records_free(r);
            if (held) {
                st = esg_bam_writer_push(wr, 0, held);
                if (st != ESG_OK) die("esg_bam_writer_push", st);
                esg_bam_records_free(held);
                held = NULL;
            }
        }
        esg_mapping_free(m);
        esg_bam_batch_free(b);
        at += n;
        ++seq;
    }
    if (held) {
        st = esg_bam_writer_push(wr, 0, held);
        if (st != ESG_OK) die("esg_bam_writer_push", st);
        esg_bam_records_free(held);
    }
    st = esg_bam_writer_close(wr);
    if (st != ESG_OK) die("esg_bam_writer_close", st);
    esg_bam_close(rd);
    if (at != counts[0]) {
        fprintf(stderr, "the mapping holds %llu reads, the BAM %llu\n",
                (unsigned long long)counts[0], (unsigned long long)at);
        return 1;
    }
    printf("records %llu\n", (unsigned long long)records);
    free(header);
    free(refs_text);
    free((void*)map);
    return 0;
}
