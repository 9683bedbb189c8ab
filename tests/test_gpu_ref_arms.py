"""The reference's own GPU kernels (comparison arms) against this library.

align_score_kernel (int) and align_score_kernel_h2 (half2), compiled ahead
of time for sm_100a from the reference's source and laid out and launched as
its GpuScorer does (oracle/ref_gpu), must give the same score for every
(query, reference) as this library's rows -- which also checks the launcher
before bench.py times it.  Skipped where the arms were not built (the
reference tree is only present where the library is built)."""
import os

import numpy as np
import pytest

from eschalign_b200 import GpuScorer, Mode, Scoring, encode, synth
from tests.helpers import Rng, random_panel, reads_for, revcomp

pytestmark = pytest.mark.gpu


def _ref_gpu(oracle, refs):
    if not (os.path.exists(oracle.REF_GPU_LIB) and os.path.exists(oracle.REF_GPU_CUBIN)):
        pytest.skip("the reference's kernels were not built (no reference tree at build time)")
    return oracle.RefGpu(refs)


@pytest.mark.parametrize("mode", [Mode.LOCAL, Mode.SEMIGLOBAL])
def test_reference_kernels_equal_our_rows(oracle, mode):
    rng = Rng(0x5EED_0A01)
    letters = random_panel(rng, 37, 20, 280)
    panel = [encode(s) for s in letters]
    reads = reads_for(rng, letters, 80)
    queries = list(reads) + [revcomp(r) for r in reads]
    scoring = (2, -1, -10, -1)
    local = mode == Mode.LOCAL
    with GpuScorer(panel, Scoring(*scoring), mode) as g:
        want = g.score_batch(reads, both_strands=True, full_rows=True).rows
    rg = _ref_gpu(oracle, panel)
    qc, qo, ql = oracle.pack(queries)
    for kernel in (0, 1):
        if rg.geometry(kernel)[0] == 0:
            continue
        got, _ = rg.score(qc, qo, ql, scoring, local, kernel=kernel)
        bad = np.argwhere(got.astype(np.int32) != want)
        assert bad.size == 0, (kernel, bad[:3], got[tuple(bad[0])], want[tuple(bad[0])])
    rg.close()


def test_reference_kernels_on_c2_sample(oracle):
    refs = synth.panel_tiles()
    reads = synth.reads_c2(refs, n=3000)
    with GpuScorer(refs, Scoring(), Mode.LOCAL) as g:
        want = g.score_batch(reads.tuple(), both_strands=True, full_rows=True).rows
    queries = reads.list() + [revcomp(r) for r in reads.list()]
    rg = _ref_gpu(oracle, refs)
    qc, qo, ql = oracle.pack(queries)
    for kernel in (0, 1):
        got, ms = rg.score(qc, qo, ql, (2, -1, -10, -1), True, kernel=kernel)
        assert np.array_equal(got.astype(np.int32), want), kernel
        assert ms > 0
    rg.close()
