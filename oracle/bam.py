"""Test infrastructure: a CPU restatement of the reference CLI's BAM output
for unpaired reads -- the records it writes for each read's mapping and their
encoding -- used as the checker of the library's BAM writer.  Nothing under
eschalign_b200/ imports it.

Restated from crates/eschalign-cli/src/align.rs:
* read_batches (align.rs:604-660): secondary and supplementary input records
  are skipped; a record aligned to the reverse strand is refused;
* process_chunk (align.rs:1504-1602): a read over --max-read-len is not
  scored and is written as an unmapped read;
* build_records (align.rs:1084-1200), OWNED_TAGS (align.rs:346-352),
  int_value (align.rs:1001-1015), sam_cigar / clipped_span
  (align.rs:1017-1052), xa_entry (align.rs:1054-1069): the output record of a
  read and, with --secondary, one record per further hit;
* the coordinate sort (align.rs:2406-2450): stable on (reference, position,
  reverse flag), unmapped last;
* the reverse complement of letters (crates/eschalign/src/alphabet.rs:69-80);
* FASTA / FASTQ input: sniff, FastxReader, normalise_seq and fastx_to_record
  (align.rs:385-563);
* paired runs: PairSource::next_pair and mate_stem (align.rs:700-870), the
  mate placements of process_pair_chunk (align.rs:1683-1713),
  build_pair_records with clipped_span / sam_cigar_ad / template_length
  (align.rs:1021-1051, 1203-1425).

The record buffer the CLI edits (noodles-sam's RecordBuf data) removes a tag
by moving its last tag into the freed slot; the new tags go to the end.  The
encoding is the BAM layout of the SAM specification (section 4.2) with its
reg2bin.  Pinned on the reference's own golden digests (unpaired_golden.tsv:
record count and FNV-1a 64 of the uncompressed record stream, as
crates/eschalign-cli/tests/align_unpaired.rs:37-62 computes them) for six
flag sets.
"""
from __future__ import annotations

import gzip
import struct

SEQ_CODES = b"=ACMGRSVTWYHKDBN"
CIGAR_CODES = {"M": 0, "I": 1, "D": 2, "N": 3, "S": 4, "H": 5, "P": 6, "=": 7, "X": 8}
OWNED_TAGS = (b"NM", b"MD", b"AS", b"XS", b"XA")  # align.rs:346-352
FLAG_REVERSE, FLAG_UNMAPPED, FLAG_SECONDARY = 0x10, 0x4, 0x100
FLAG_QC_FAIL, FLAG_DUPLICATE, FLAG_SUPPLEMENTARY = 0x200, 0x400, 0x800
_AUX_SIZE = {b"A": 1, b"c": 1, b"C": 1, b"s": 2, b"S": 2, b"i": 4, b"I": 4, b"f": 4}


def split_aux(b: bytes):
    """[(tag, encoded field bytes)] of a BAM record's auxiliary data."""
    out, i = [], 0
    while i < len(b):
        tag, t = b[i:i + 2], b[i + 2:i + 3]
        j = i + 3
        if t in _AUX_SIZE:
            j += _AUX_SIZE[t]
        elif t in (b"Z", b"H"):
            j = b.index(b"\0", j) + 1
        elif t == b"B":
            n = struct.unpack("<I", b[j + 1:j + 5])[0]
            j += 5 + n * _AUX_SIZE[b[j:j + 1]]
        else:
            raise ValueError(f"unknown aux type {t!r}")
        out.append((tag, b[i:j]))
        i = j
    return out


def read_bam(data: bytes):
    """(header text, [(name, length)], records) of a BGZF-compressed BAM;
    a record is a dict of its flag, name, sequence letters, qualities and
    (tag, field bytes) auxiliary list."""
    raw = gzip.decompress(data)
    if raw[:4] != b"BAM\1":
        raise ValueError("not a BAM file")
    lt = struct.unpack("<I", raw[4:8])[0]
    text = raw[8:8 + lt]
    o = 8 + lt
    n_ref = struct.unpack("<I", raw[o:o + 4])[0]
    o += 4
    refs = []
    for _ in range(n_ref):
        ln = struct.unpack("<I", raw[o:o + 4])[0]
        name = raw[o + 4:o + 4 + ln - 1]
        refs.append((name, struct.unpack("<I", raw[o + 4 + ln:o + 8 + ln])[0]))
        o += 8 + ln
    recs = []
    while o < len(raw):
        bs = struct.unpack("<I", raw[o:o + 4])[0]
        r = raw[o + 4:o + 4 + bs]
        o += 4 + bs
        (_, _, lrn, _, _, ncig, flag, lseq, _, _, _) = struct.unpack("<iiBBHHHIiii", r[:32])
        p = 32
        name = r[p:p + lrn - 1]
        p += lrn + 4 * ncig
        sb = r[p:p + (lseq + 1) // 2]
        p += (lseq + 1) // 2
        seq = bytes(SEQ_CODES[(sb[k // 2] >> (0 if k % 2 else 4)) & 0xF] for k in range(lseq))
        qual = r[p:p + lseq]
        p += lseq
        recs.append({"flag": flag, "name": name, "seq": seq, "qual": qual,
                     "aux": split_aux(r[p:])})
    return text, refs, recs


def input_reads(recs):
    """read_batches (align.rs:604-660): the primary records, in order."""
    out = []
    for r in recs:
        if r["flag"] & (FLAG_SECONDARY | FLAG_SUPPLEMENTARY):
            continue
        if not r["flag"] & FLAG_UNMAPPED and r["flag"] & FLAG_REVERSE:
            raise ValueError("input record aligned to the reverse strand")
        out.append(r)
    return out


_ASCII_WS = b" \t\n\x0c\r"  # Rust's u8::is_ascii_whitespace


def sniff(data: bytes) -> str:
    """sniff (align.rs:385-414): "bam", "fasta" or "fastq"."""
    gz = data[:2] == b"\x1f\x8b"
    payload = gzip.decompress(data) if gz else data
    if payload[:4] == b"BAM\1":
        if not gz:
            raise ValueError("uncompressed BAM is not supported")
        return "bam"
    first = payload.lstrip(_ASCII_WS)[:1]
    if first == b">":
        return "fasta"
    if first == b"@":
        return "fastq"
    raise ValueError("not a BAM, FASTA or FASTQ file (plain or gzip)")


def normalise_seq(seq: bytes) -> bytes:
    """normalise_seq (align.rs:539-549): upper case, U as T, anything outside
    the BAM alphabet as N."""
    out = bytearray()
    for b in seq.upper():
        out.append(ord("T") if b == ord("U") else (b if b in SEQ_CODES else ord("N")))
    return bytes(out)


def read_fastx(data: bytes):
    """FastxReader::next_record (align.rs:436-537) over a whole FASTA / FASTQ
    file (plain or gzip), each record as fastx_to_record (align.rs:551-563)
    makes it: an unmapped record in read_bam's form (no tags; FASTQ
    qualities Phred + 33 saturating at 0, FASTA ones missing)."""
    fastq = sniff(data) == "fastq"
    text = gzip.decompress(data) if data[:2] == b"\x1f\x8b" else data
    lines = text.split(b"\n")
    if lines and lines[-1] == b"":
        lines.pop()  # the terminator of the last line
    lines = [ln.rstrip(b"\r\n") for ln in lines]

    def name_of(h):
        for k, b in enumerate(h):
            if b in _ASCII_WS:
                return h[:k]
        return h
    out, i = [], 0
    while True:
        while i < len(lines) and lines[i] == b"":
            i += 1
        if i == len(lines):
            return out
        h = lines[i]
        i += 1
        if h[:1] != (b"@" if fastq else b">"):
            raise ValueError(f"line {i}: expected {'@' if fastq else '>'}")
        name = name_of(h[1:])
        if fastq:
            if i >= len(lines):
                raise ValueError("FASTQ truncated after header")
            if i + 1 >= len(lines) or lines[i + 1][:1] != b"+":
                raise ValueError("FASTQ: expected '+'")
            if i + 2 >= len(lines):
                raise ValueError("FASTQ truncated before quality")
            seq, qual = lines[i], lines[i + 2]
            if len(qual) != len(seq):
                raise ValueError("FASTQ: quality and sequence lengths differ")
            i += 3
            q = bytes(max(c - 33, 0) for c in qual)
        else:
            seq = bytearray()
            while i < len(lines) and lines[i][:1] != b">":
                seq += bytes(b for b in lines[i] if b not in _ASCII_WS)
                i += 1
            seq, q = bytes(seq), b""
        out.append({"flag": FLAG_UNMAPPED, "name": name, "seq": normalise_seq(seq),
                    "qual": q, "aux": []})


def reg2bin(beg: int, end: int) -> int:
    """The SAM specification's bin of [beg, end) (0-based, end exclusive)."""
    end -= 1
    for shift, base in ((14, 4681), (17, 585), (20, 73), (23, 9), (26, 1)):
        if beg >> shift == end >> shift:
            return base + (beg >> shift)
    return 0


def int_field(tag: bytes, v: int) -> bytes:
    """int_value (align.rs:1001-1015): the smallest of u8, i8, u16, i16, u32,
    else i32."""
    for code, fmt, lo, hi in ((b"C", "<B", 0, 255), (b"c", "<b", -128, 127),
                              (b"S", "<H", 0, 65535), (b"s", "<h", -32768, 32767),
                              (b"I", "<I", 0, 2**32 - 1)):
        if lo <= v <= hi:
            return tag + code + struct.pack(fmt, v)
    return tag + b"i" + struct.pack("<i", v)


def str_field(tag: bytes, s: str) -> bytes:
    return tag + b"Z" + s.encode() + b"\0"


def encode_record(refid, pos, mapq, cigar, flag, name, seq, qual, aux, mate_ref=-1, mate_pos=-1,
                  tlen=0) -> bytes:
    """One BAM record (block_size included); cigar is [(length, op)], pos
    0-based or -1, aux the encoded fields in order.  The bin is noodles'
    (the writer of the CLI): the region [pos, pos + span - 1], so a record
    with a position and no CIGAR (an unmapped mate placed at its partner's
    position) takes the bin of [pos, pos - 1], and none (4680) at pos 0."""
    span = sum(n for n, op in cigar if op in "MDN=X")
    if pos < 0 or (span == 0 and pos == 0):
        b = 4680
    else:
        b = reg2bin(pos, pos + span)
    nm = (name if name else b"*") + b"\0"
    body = struct.pack("<iiBBHHHIiii", refid, pos, len(nm), mapq, b, len(cigar), flag, len(seq),
                       mate_ref, mate_pos, tlen)
    body += nm + b"".join(struct.pack("<I", n << 4 | CIGAR_CODES[op]) for n, op in cigar)
    sb = bytearray((len(seq) + 1) // 2)
    for k, ch in enumerate(seq):
        c = SEQ_CODES.find(bytes([ch]).upper())
        sb[k // 2] |= (c if c >= 0 else 15) << (0 if k % 2 else 4)
    body += bytes(sb) + (qual if len(qual) == len(seq) else b"\xff" * len(seq)) + b"".join(aux)
    return struct.pack("<I", len(body)) + body


def revcomp_letters(s: bytes) -> bytes:
    """alphabet::reverse_complement (alphabet.rs:69-80)."""
    m = {ord("A"): b"T", ord("C"): b"G", ord("G"): b"C", ord("T"): b"A", ord("U"): b"A"}
    return b"".join(m.get(c, b"N") for c in bytes(s).upper()[::-1])


def _cigar_ops(s: str):
    out, n = [], ""
    for ch in s:
        if ch.isdigit():
            n += ch
        else:
            out.append((int(n), ch))
            n = ""
    return out


def _without_owned(aux, tags=OWNED_TAGS):
    """RecordBuf data with `tags` removed, in that order: each removal moves
    the last tag into the freed slot."""
    aux = list(aux)
    for t in tags:
        for i, (tag, _) in enumerate(aux):
            if tag == t:
                last = aux.pop()
                if i < len(aux):
                    aux[i] = last
                break
    return aux


def build_records(rec, m, ref_names, secondary=False):
    """build_records (align.rs:1084-1200) for one read and its mapping (the
    oracle's map_reads form: best_score, n_tied, suboptimal, hits)."""
    kept = rec["flag"] & (FLAG_QC_FAIL | FLAG_DUPLICATE)
    aux = _without_owned(rec["aux"])
    hits = m["hits"]
    if not hits:
        return [encode_record(-1, -1, 0, [], kept | FLAG_UNMAPPED, rec["name"], rec["seq"],
                              rec["qual"], [f for _, f in aux])]
    n = len(rec["seq"])

    def sam_cigar(h):  # sam_cigar / clipped_span (align.rs:1017-1052)
        c = [(h["query_start"], "S")] if h["query_start"] > 0 else []
        c += _cigar_ops(h["cigar"])
        if n > h["query_end"]:
            c.append((n - h["query_end"], "S"))
        return c

    p = hits[0]
    seq, qual, flag = rec["seq"], rec["qual"], kept
    if p["reverse"]:
        flag |= FLAG_REVERSE
        seq, qual = revcomp_letters(seq), qual[::-1]
    fields = [f for _, f in aux]
    fields += [int_field(b"NM", p["nm"]), str_field(b"MD", p["md"]),
               int_field(b"AS", m["best_score"])]
    if m["suboptimal"] is not None:
        fields.append(int_field(b"XS", m["suboptimal"]))
    if len(hits) > 1:  # xa_entry (align.rs:1054-1069)
        xa = "".join(f"{ref_names[h['reference']]},{'-' if h['reverse'] else '+'}"
                     f"{h['ref_start'] + 1},{''.join(f'{k}{op}' for k, op in sam_cigar(h))},"
                     f"{h['nm']};" for h in hits[1:])
        fields.append(str_field(b"XA", xa))
    out = [encode_record(p["reference"], p["ref_start"], 60 if m["n_tied"] == 1 else 0,
                         sam_cigar(p), flag, rec["name"], seq, qual, fields)]
    if secondary:
        rg = [f for t, f in rec["aux"] if t == b"RG"][:1]  # the first, as Data::get finds it
        for h in hits[1:]:
            d = [int_field(b"NM", h["nm"]), str_field(b"MD", h["md"]),
                 int_field(b"AS", m["best_score"])] + rg
            out.append(encode_record(h["reference"], h["ref_start"], 0, sam_cigar(h),
                                     FLAG_SECONDARY | kept | (FLAG_REVERSE if h["reverse"] else 0),
                                     rec["name"], b"", b"", d))
    return out


# ---------------------------------------------------------------- pairs
FLAG_PAIRED, FLAG_PROPER, FLAG_MATE_UNMAPPED = 0x1, 0x2, 0x8
FLAG_MATE_REVERSE, FLAG_FIRST, FLAG_LAST = 0x20, 0x40, 0x80
PAIR_OWNED_TAGS = OWNED_TAGS + (b"MC", b"ad")  # align.rs:1203-1206, 1262


def canonical_read_name(name: bytes) -> bytes:
    """canonical_read_name (align.rs:572-583) with parse_uuid_flexible
    (uuid_util.rs:10-30): a UUID name, in any spelling the uuid crate parses
    (32 hex digits, dashed, braced, urn:uuid:), as its dashed lower-case
    form; any other name as it is."""
    import re
    s = name.decode("latin-1")
    m = (re.fullmatch(r"[0-9a-fA-F]{32}", s)
         or re.fullmatch(r"(?:\{|urn:uuid:)?([0-9a-fA-F]{8})-([0-9a-fA-F]{4})-([0-9a-fA-F]{4})-"
                         r"([0-9a-fA-F]{4})-([0-9a-fA-F]{12})\}?", s))
    if not m or (s.startswith("{") != s.endswith("}")) or (s.startswith("urn:") and
                                                         s.endswith("}")):
        return name
    h = "".join(m.groups()) if m.groups() else s
    h = h.lower()
    return f"{h[:8]}-{h[8:12]}-{h[12:16]}-{h[16:20]}-{h[20:]}".encode()


def load_read_ids(text: bytes):
    """load_read_ids (align.rs:585-601): the canonical names of an ID list."""
    ids = set()
    for line in text.split(b"\n"):
        line = line.strip(_ASCII_WS)
        if line and not line.startswith(b"#"):
            ids.add(canonical_read_name(line.split()[0]))
    if not ids:
        raise ValueError("no read names")
    return ids


def select_reads(recs, wanted):
    """read_batches' --read-ids filter (align.rs:611-621): a record without
    a name ('*') is not kept."""
    return [r for r in recs
            if r["name"] != b"*" and canonical_read_name(r["name"]) in wanted]


def mate_stem(name: bytes) -> bytes:
    """mate_stem (align.rs:700-706): the name without a trailing /1 or /2."""
    return name[:-2] if len(name) >= 2 and name[-2:] in (b"/1", b"/2") else name


def _renamed(rec, name):
    r = dict(rec)
    r["name"] = name
    return r


def read_pairs(data1: bytes, data2: bytes | None = None, wanted=None):
    """read_pair_batches (align.rs:875-905): the pairs of _read_pairs, with
    --read-ids (`wanted`, canonical names) selecting by the pair's name."""
    pairs = _read_pairs(data1, data2)
    if wanted is None:
        return pairs
    return [(a, b) for a, b in pairs if canonical_read_name(a["name"]) in wanted]


def _read_pairs(data1: bytes, data2: bytes | None = None):
    """PairSource::next_pair (align.rs:759-870): [(mate 1, mate 2)] of two
    FASTA / FASTQ files, one interleaved FASTX file, or a paired BAM (mates
    adjacent, 0x1 with one of 0x40 / 0x80), each mate named by the pair's
    stem (process_pair_chunk, align.rs:1631-1639).  Errors raise ValueError
    naming the read."""
    out = []
    if data2 is not None:
        a, b = read_fastx(data1), read_fastx(data2)
        for k in range(max(len(a), len(b))):
            if k >= len(b):
                raise ValueError(f"read {a[k]['name'].decode()} has no mate")
            if k >= len(a):
                raise ValueError(f"read {b[k]['name'].decode()} has no mate")
            if mate_stem(a[k]["name"]) != mate_stem(b[k]["name"]):
                raise ValueError(f"mate names differ: {a[k]['name'].decode()} but "
                                 f"{b[k]['name'].decode()}")
            stem = mate_stem(a[k]["name"])
            out.append((_renamed(a[k], stem), _renamed(b[k], stem)))
        return out
    if sniff(data1) != "bam":
        recs = read_fastx(data1)
        for k in range(0, len(recs), 2):
            if k + 1 >= len(recs):
                raise ValueError(f"read {recs[k]['name'].decode()} has no mate")
            x, y = recs[k], recs[k + 1]
            if mate_stem(x["name"]) != mate_stem(y["name"]):
                raise ValueError(f"read {x['name'].decode()} has no mate: the next record is "
                                 f"{y['name'].decode()}")
            stem = mate_stem(x["name"])
            out.append((_renamed(x, stem), _renamed(y, stem)))
        return out
    _, _, recs = read_bam(data1)
    recs = input_reads(recs)
    for k in range(0, len(recs), 2):
        x = recs[k]
        fx = x["flag"]
        if not fx & FLAG_PAIRED or bool(fx & FLAG_FIRST) == bool(fx & FLAG_LAST):
            raise ValueError(f"read {x['name'].decode()}: not a mate")
        if k + 1 >= len(recs):
            raise ValueError(f"read {x['name'].decode()} has no mate")
        y = recs[k + 1]
        fy = y["flag"]
        if mate_stem(x["name"]) != mate_stem(y["name"]):
            raise ValueError(f"read {x['name'].decode()} has no mate: the next record is "
                             f"{y['name'].decode()}")
        if (not fy & FLAG_PAIRED or bool(fy & FLAG_FIRST) == bool(fy & FLAG_LAST)
                or bool(fy & FLAG_FIRST) == bool(fx & FLAG_FIRST)):
            raise ValueError(f"read {mate_stem(x['name']).decode()}: not mate 1 and mate 2")
        stem = mate_stem(x["name"])
        m1, m2 = (x, y) if fx & FLAG_FIRST else (y, x)
        out.append((_renamed(m1, stem), _renamed(m2, stem)))
    return out


def clipped_span(h, ad):
    """clipped_span (align.rs:1021-1029): the aligned part within the whole
    SEQ, the adapter being the 3' end (the start of a reverse hit's SEQ)."""
    shift = ad if h["reverse"] else 0
    return h["query_start"] + shift, h["query_end"] + shift


def sam_cigar_ad(h, full, ad):
    """sam_cigar_ad (align.rs:1031-1051) as [(length, op)]."""
    qs, qe = clipped_span(h, ad)
    c = [(qs, "S")] if qs > 0 else []
    c += _cigar_ops(h["cigar"])
    if full > qe:
        c.append((full - qe, "S"))
    return c


def _cigar_text(c):
    return "".join(f"{n}{op}" for n, op in c)


def template_length(h, partner, first):
    """template_length (align.rs:1225-1236)."""
    n = max(h["ref_end"], partner["ref_end"]) - min(h["ref_start"], partner["ref_start"])
    left = h["ref_start"] < partner["ref_start"] or (h["ref_start"] == partner["ref_start"]
                                                     and first)
    return n if left else -n


def pair_placements(pm):
    """process_pair_chunk's MatePlacement per mate (align.rs:1683-1713) from
    the oracle's map_pairs form; returns (placements, proper)."""
    if pm["proper"]:
        hits = pm["hits"]
        return [{"primary": hits[0]["mates"][m],
                 "others": [h["mates"][m] for h in hits[1:]],
                 "partners": [h["mates"][1 - m] for h in hits[1:]],
                 "score": hits[0]["mates"][m]["score"], "xs": pm["suboptimal"][m],
                 "unique": pm["n_tied"] == 1} for m in range(2)], True
    ms = pm["mates"]
    out = []
    for m in range(2):
        me, other = ms[m], ms[1 - m]
        others = me["hits"][1:]
        out.append({"primary": me["hits"][0] if me["hits"] else None, "others": others,
                    "partners": [other["hits"][0] if other["hits"] else None] * len(others),
                    "score": me["best_score"] if me["best_score"] is not None else 0,
                    "xs": me["suboptimal"], "unique": me["n_tied"] == 1})
    return out, False


def build_pair_records(recs, pm, ad, ref_names, secondary=False):
    """build_pair_records (align.rs:1238-1425) for one pair: [mate 1, mate 2,
    then with `secondary` a pair of 0x100 records per further tie-set
    member]; `ad` is [mate 1, mate 2] adapter bases, or None when adapters
    were not searched (no `ad` tag)."""
    place, proper = pair_placements(pm)
    full = [len(recs[0]["seq"]), len(recs[1]["seq"])]
    adn = ad if ad is not None else [0, 0]
    seg = [FLAG_FIRST, FLAG_LAST]
    st = []
    for m in range(2):
        r = recs[m]
        kept = r["flag"] & (FLAG_QC_FAIL | FLAG_DUPLICATE)
        fields = [f for _, f in _without_owned(r["aux"], PAIR_OWNED_TAGS)]
        d = {"kept": kept, "flag": kept | FLAG_PAIRED | seg[m], "ref": -1, "pos": -1, "mapq": 0,
             "cigar": [], "seq": r["seq"], "qual": r["qual"], "fields": fields,
             "mate_ref": -1, "mate_pos": -1, "tlen": 0}
        h = place[m]["primary"]
        if h is None:
            d["flag"] |= FLAG_UNMAPPED
        else:
            if h["reverse"]:
                d["flag"] |= FLAG_REVERSE
                d["seq"], d["qual"] = revcomp_letters(r["seq"]), r["qual"][::-1]
            d["ref"], d["pos"] = h["reference"], h["ref_start"]
            d["mapq"] = 60 if place[m]["unique"] else 0
            d["cigar"] = sam_cigar_ad(h, full[m], adn[m])
            fields += [int_field(b"NM", h["nm"]), str_field(b"MD", h["md"]),
                       int_field(b"AS", place[m]["score"])]
            if place[m]["xs"] is not None:
                fields.append(int_field(b"XS", place[m]["xs"]))
            if place[m]["others"]:
                fields.append(str_field(b"XA", "".join(
                    f"{ref_names[o['reference']]},{'-' if o['reverse'] else '+'}"
                    f"{o['ref_start'] + 1},{_cigar_text(sam_cigar_ad(o, full[m], adn[m]))},"
                    f"{o['nm']};" for o in place[m]["others"])))
        if ad is not None:
            fields.append(int_field(b"ad", ad[m]))
        st.append(d)
    for m in range(2):
        o = 1 - m
        h, oh, d = place[m]["primary"], place[o]["primary"], st[m]
        if h is not None and oh is not None:
            if oh["reverse"]:
                d["flag"] |= FLAG_MATE_REVERSE
            if proper:
                d["flag"] |= FLAG_PROPER
            d["mate_ref"], d["mate_pos"] = oh["reference"], oh["ref_start"]
            d["fields"].append(str_field(b"MC", _cigar_text(sam_cigar_ad(oh, full[o], adn[o]))))
            if h["reference"] == oh["reference"]:
                d["tlen"] = template_length(h, oh, m == 0)
        elif h is not None:
            d["flag"] |= FLAG_MATE_UNMAPPED
            d["mate_ref"], d["mate_pos"] = h["reference"], h["ref_start"]
        elif oh is not None:
            if oh["reverse"]:
                d["flag"] |= FLAG_MATE_REVERSE
            d["ref"], d["pos"] = oh["reference"], oh["ref_start"]
            d["mate_ref"], d["mate_pos"] = oh["reference"], oh["ref_start"]
        else:
            d["flag"] |= FLAG_MATE_UNMAPPED
    out = [encode_record(d["ref"], d["pos"], d["mapq"], d["cigar"], d["flag"], recs[m]["name"],
                         d["seq"], d["qual"], d["fields"], d["mate_ref"], d["mate_pos"], d["tlen"])
           for m, d in enumerate(st)]
    if secondary:
        for k in range(max(len(place[0]["others"]), len(place[1]["others"]))):
            for m in range(2):
                if k >= len(place[m]["others"]):
                    continue
                h, ph = place[m]["others"][k], place[m]["partners"][k]
                f = FLAG_SECONDARY | FLAG_PAIRED | seg[m] | st[m]["kept"]
                if h["reverse"]:
                    f |= FLAG_REVERSE
                fields = [int_field(b"NM", h["nm"]), str_field(b"MD", h["md"]),
                          int_field(b"AS", h["score"])]
                fields += [fl for t, fl in recs[m]["aux"] if t == b"RG"][:1]
                mref, mpos, tlen = h["reference"], h["ref_start"], 0
                if ph is not None:
                    if ph["reverse"]:
                        f |= FLAG_MATE_REVERSE
                    mref, mpos = ph["reference"], ph["ref_start"]
                    if proper:
                        f |= FLAG_PROPER
                        if ph["reference"] == h["reference"]:
                            tlen = template_length(h, ph, m == 0)
                else:
                    f |= FLAG_MATE_UNMAPPED
                out.append(encode_record(h["reference"], h["ref_start"], 0,
                                         sam_cigar_ad(h, full[m], adn[m]), f, recs[m]["name"],
                                         b"", b"", fields, mref, mpos, tlen))
    return out


def coordinate_order(records):
    """The coordinate sort (align.rs:2406-2450): stable on (reference,
    position, reverse), unmapped last."""
    def key(r):
        tid, pos = struct.unpack("<ii", r[4:12])
        flag = struct.unpack("<H", r[18:20])[0]
        return (tid if tid >= 0 else 1 << 40, pos, bool(flag & FLAG_REVERSE))
    return sorted(records, key=key)


def fnv1a64(b: bytes) -> int:
    """The digest of crates/eschalign-cli/tests/align_unpaired.rs:37-62."""
    h = 0xCBF29CE484222325
    for x in b:
        h = ((h ^ x) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h
