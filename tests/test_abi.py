"""The C-ABI library builds for sm_100a, loads without a GPU, and exports
every entry point include/eschalign_b200.h declares (no compute here)."""
import ctypes
import os
import re

import pytest

import eschalign_b200
from eschalign_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "eschalign_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(esg_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_bound_api():
    names = declared()
    assert "esg_scorer_new" in names and "esg_score_batch" in names
    assert set(names) == set(_native.SIGNATURES), set(names) ^ set(_native.SIGNATURES)


def test_library_loads_and_exports_every_symbol():
    lib = eschalign_b200.load()
    for name in declared():
        assert hasattr(lib, name), name
    assert lib.esg_abi_version() == 1
    assert lib.esg_status_string(0) == b"ok"


def test_no_device_is_an_error_not_a_crash():
    """GpuScorer::new returns Unavailable without a device (cuda/mod.rs:356-366)."""
    import numpy as np
    from eschalign_b200 import GpuError, GpuScorer, Mode, Scoring, device_visible
    if device_visible():
        pytest.skip("a device is present")
    with pytest.raises(GpuError) as ei:
        GpuScorer([np.array([0, 1, 2, 3], np.uint8)], Scoring(), Mode.LOCAL)
    assert ei.value.kind == "Unavailable"


def _new(lib, refs, scoring=(2, -1, -10, -1), mode=0, cap=8):
    import numpy as np
    lens = np.array([len(r) for r in refs], dtype=np.uint32)
    off = np.zeros(len(refs), dtype=np.uint64)
    if len(refs) > 1:
        off[1:] = np.cumsum(lens[:-1])
    codes = np.concatenate([np.asarray(r, np.uint8) for r in refs] + [np.zeros(1, np.uint8)])
    sc = _native.EsgScoring(*scoring)
    opts = _native.EsgOptions(cap, 0, None)
    h = ctypes.c_void_p()
    P = lambda a, t: a.ctypes.data_as(ctypes.POINTER(t))
    return lib.esg_scorer_new(0, P(codes, ctypes.c_uint8), P(off, ctypes.c_uint64),
                              P(lens, ctypes.c_uint32), len(refs), ctypes.byref(sc), mode,
                              ctypes.byref(opts), ctypes.byref(h))


def test_argument_refusals_before_any_device_call():
    """Panel and scoring refusals (panel.rs:34-55, scoring.rs:70-100,
    cuda/mod.rs:367-373) come back as status codes, on any host."""
    import numpy as np
    lib = eschalign_b200.load()
    ok = [np.array([0, 1, 2, 3], np.uint8)]
    assert _new(lib, []) == 5                                   # EmptyPanel
    assert _new(lib, [np.zeros(0, np.uint8)]) == 6              # EmptyReference
    assert _new(lib, [np.zeros(32769, np.uint8)]) == 3          # ReferenceTooLong
    assert _new(lib, ok, scoring=(0, -1, -10, -1)) == 4         # ScoringInvalid
    assert _new(lib, ok, scoring=(2, 3, -10, -1)) == 4
    assert _new(lib, ok, scoring=(2, -1, 5, -1)) == 4
    assert _new(lib, ok, scoring=(2, -1, -1001, -1)) == 4
    assert _new(lib, ok, mode=7) == 7                           # BadArgument
    assert _new(lib, ok, cap=33) == 7
    assert b"exceeds" in lib.esg_last_error() or lib.esg_last_error()


def test_mapping_entry_points_refuse_bad_arguments_on_any_host():
    """esg_map_reads / esg_map_pairs check their arguments before touching a
    scorer or a device; the mapping accessors take NULL."""
    import ctypes
    import numpy as np
    from eschalign_b200 import _native
    lib = eschalign_b200.load()
    out = ctypes.c_void_p(123)
    mo = _native.EsgMapOptions(0, 0xFFFFFFFF, 0, 0)
    po = _native.EsgPairMapOptions(0, 0xFFFFFFFF, 500, 0)
    lens = np.array([4], np.uint32)
    off = np.array([0], np.uint64)
    u32 = ctypes.POINTER(ctypes.c_uint32)
    u64 = ctypes.POINTER(ctypes.c_uint64)
    assert lib.esg_map_reads(None, None, None, None, 0, ctypes.byref(mo), None, None,
                             ctypes.byref(out)) == 7
    assert out.value is None                                    # cleared on refusal
    assert lib.esg_map_pairs(None, None, None, None, 0, ctypes.byref(po), None, None,
                             ctypes.byref(out)) == 7
    fake = ctypes.c_void_p(1)  # never dereferenced: the options are refused first
    assert lib.esg_map_reads(fake, None, off.ctypes.data_as(u64), lens.ctypes.data_as(u32), 1,
                             None, None, None, ctypes.byref(out)) == 7
    n32, n64 = ctypes.c_uint32(9), ctypes.c_uint64(9)
    assert lib.esg_mapping_reads(None, ctypes.byref(n32)) is None and n32.value == 0
    assert lib.esg_mapping_hits(None, ctypes.byref(n64)) is None and n64.value == 0
    assert lib.esg_mapping_pairs(None, ctypes.byref(n32)) is None and n32.value == 0
    assert lib.esg_mapping_pair_hits(None, ctypes.byref(n64)) is None
    lib.esg_mapping_free(None)


# ctypes mirror -> the header's struct name
_STRUCTS = {"EsgScoring": "esg_scoring", "EsgOptions": "esg_options", "EsgInfo": "esg_info",
            "EsgTuneReport": "esg_tune_report", "EsgBatchStats": "esg_batch_stats",
            "EsgAdapterConfig": "esg_adapter_config", "EsgAlignJob": "esg_align_job",
            "EsgAlignment": "esg_alignment", "EsgMapOptions": "esg_map_options",
            "EsgPairMapOptions": "esg_pair_map_options", "EsgServerOptions": "esg_server_options",
            "EsgRequestTiming": "esg_request_timing", "EsgServerStats": "esg_server_stats"}


def test_ctypes_structs_match_the_header(tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler
    gives the header's struct (a drifted mirror would read garbage)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"',
             "int main(void) {"]
    for py, c in _STRUCTS.items():
        lines.append(f'printf("{py} size %zu\\n", sizeof({c}));')
        for fname, _ in getattr(_native, py)._fields_:
            lines.append(f'printf("{py} {fname} %zu\\n", offsetof({c}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run([cc, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        py, what, val = line.split()
        cls = getattr(_native, py)
        got = ctypes.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert got == int(val), (py, what, got, val)
