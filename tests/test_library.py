"""The C-ABI library on the CPU: it loads without a GPU and exports every function include/*.h declares
(no compute call is made here)."""

import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBRARY = os.path.join(ROOT, "dinara-align_b200", "dinara_align", "libdinara_gpu.so")


def declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for match in re.finditer(r"^[A-Za-z_][\w \*]*?\b(dinara_\w+)\s*\(", text, flags=re.M):
            names.add(match.group(1))
    return names


def test_library_exports_every_declared_function():
    assert os.path.exists(LIBRARY), "build the library first (make -C dinara-align_b200)"
    handle = ctypes.CDLL(LIBRARY)
    names = declared_functions()
    assert len(names) >= 10
    missing = [name for name in sorted(names) if not hasattr(handle, name)]
    assert not missing, missing


def test_null_context_is_refused():
    """A call without a context fails with a code, not a crash, and touches no device."""
    handle = ctypes.CDLL(LIBRARY)
    handle.dinara_gpu_scores_tape.restype = ctypes.c_int64
    code = handle.dinara_gpu_scores_tape(None, 0, None, None, None, None, None, None)
    assert code == -6
    handle.dinara_free.restype = None
    handle.dinara_free(None)


def test_python_package_imports_without_gpu():
    import sys

    sys.path.insert(0, os.path.join(ROOT, "dinara-align_b200"))
    import dinara_align

    assert dinara_align.Scoring.dna().table[0] == 2
    assert dinara_align.Tape.of(["AC"], ["G"]).pairs == 1
    assert dinara_align.Costs.edit().unit_scale() == 1
    assert dinara_align.Costs.affine(4, 6, 2).unit_scale() == 0


def test_sam_fields():
    """An alignment's SAM fields from its CIGAR and span, with the reference's own answers
    (tests/test_python.py:89-91): the clipped CIGAR, MD and NM."""
    import dinara_align as da

    core = da.Alignment(0, 14, "4=1X3=", 4, 12, 4, 12)
    assert core.clipped_cigar(14) == "4S4=1X3=2S"
    assert core.clipped_cigar(14, hard=True) == "4H4=1X3=2H"
    assert core.mismatch_string("GGGGACGTACGTGGGG", "CCCCACGTTCGTCC") == "4A3"
    assert core.edit_distance("GGGGACGTACGTGGGG", "CCCCACGTTCGTCC") == 1
    gapped = da.Alignment(2, -2, "2=2D2=1I1=", 0, 7, 0, 6)
    assert gapped.gapped("ACGTTGA", "ACTGCA") == ("ACGTTG-A", "AC--TGCA")
    assert gapped.mismatch_string("ACGTTGA", "ACTGCA") == "2^GT3"
    assert gapped.edit_distance("ACGTTGA", "ACTGCA") == 3
    assert da.Costs.affine(4, 6, 2).with_deletions(20, 5).unit_scale() == 0 and da.Costs.linear(3, 3).unit_scale() == 3


def test_band_tuning_needs_a_context():
    """The autotuner's entry points refuse a missing context with a code."""
    handle = ctypes.CDLL(LIBRARY)
    handle.dinara_gpu_band_tuning.restype = ctypes.c_int64
    values = (ctypes.c_byte * 256)()
    assert handle.dinara_gpu_band_tuning(None, 0, values) == -6
    handle.dinara_gpu_band_autotune.restype = ctypes.c_int64
    assert handle.dinara_gpu_band_autotune(None, None, None) == -6


def test_tuning_for_each_start():
    """An autotune report's per-candidate times split into plain doubling's and the near starts' parts: each
    start takes the bound fastest for it, the measured word costs and grid scheme kept."""
    from dinara_align import tuning

    report = {"chain_ms": {"24000/0/5": 120.0, "48000/0/5": 113.0, "24000/1/8": 118.0},
              "chain_ms_near": {"24000/0/5": 41.5, "48000/0/5": 40.6, "24000/1/8": 48.2}}
    values = {"chain_words": 48000, "chain_share": 0.0, "reach": 5, "full_grids": 0, "word_costs": [40.0] * 39}
    near = tuning.tuning_for_starts(report, values, near=True)
    plain = tuning.tuning_for_starts(report, values, near=False)
    assert (near["chain_words"], near["chain_share"], near["reach"]) == (48000, 0.0, 5)
    assert (plain["chain_words"], plain["chain_share"], plain["reach"]) == (24000, 1.0, 8)
    assert plain["word_costs"] == values["word_costs"] and plain["full_grids"] == 0
