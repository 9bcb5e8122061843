"""Writes tests/golden/known_answers.json and tests/golden/random_pairs.json.

known_answers.json holds the reference's own known answers for this path, transcribed from its tests
(each entry names the reference file and line it comes from). random_pairs.json holds seeded pairs made
by the reference's Python test generator's rules (tests/test_python.py:26-43 `mutated`, random.Random(7),
reference lengths 0-119, error rates 0/5/20/50% in turn), with their unit-cost distance by a plain
dynamic program (the one tests/test_python.py:16-23 checks against) and their Gotoh scores and CIGARs by
the CPU oracle (oracle/), as regression fixtures for the GPU tests.

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))

import oracle  # noqa: E402

DNA = {"alphabet": "ACGT", "table": [2 if r == c else -4 for r in range(4) for c in range(4)], "opening": -4,
       "extension": -2}
CONFIG2 = {"alphabet": "ACGT", "table": [0 if r == c else -4 for r in range(4) for c in range(4)], "opening": -6,
           "extension": -2}
TABULATED = {"alphabet": "ACGT", "table": [5, -1, -2, -1, -1, 5, -3, -2, -2, -3, 5, -1, -1, -2, -1, 5], "opening": -6,
             "extension": -1}

KNOWN = [
    # Scoring path, global (tests/test_alignment.mojo:304-331; the CIGARs are the reference's host walk's,
    # which the GPU walk matches on these pairs).
    {"kind": "score", "reference": "ACGTACGT", "query": "ACGTACGT", "scoring": DNA, "mode": "global", "score": 16,
     "cigar": "8=", "source": "tests/test_alignment.mojo:304-308"},
    {"kind": "score", "reference": "ACGTACGT", "query": "ACGTTCGT", "scoring": DNA, "mode": "global", "score": 10,
     "cigar": "4=1X3=", "cigar_m": "8M", "source": "tests/test_alignment.mojo:310-314, 323-324"},
    {"kind": "score", "reference": "ACGTTGCAGGGCATGACGT", "query": "ACGTTGCACATGACGT", "scoring": DNA,
     "mode": "global", "score": 22, "cigar": "8=3D8=", "source": "tests/test_alignment.mojo:316-326"},
    {"kind": "score", "reference": "AAAA", "query": "", "scoring": DNA, "mode": "global", "score": -12,
     "source": "tests/test_alignment.mojo:329"},
    {"kind": "score", "reference": "", "query": "", "scoring": DNA, "mode": "global", "score": 0,
     "source": "tests/test_alignment.mojo:330"},
    # Scoring path, local (tests/test_alignment.mojo:333-341; tests/test_python.py:96).
    {"kind": "score", "reference": "GGGGACGTACGTGGGG", "query": "CCCCACGTACGTCCCC", "scoring": DNA, "mode": "local",
     "score": 16, "cigar": "8=", "reference_start": 4, "query_end": 12, "source": "tests/test_alignment.mojo:333-341"},
    {"kind": "score", "reference": "TTTTACGTACGTTTTT", "query": "ACGTACGT", "scoring": DNA, "mode": "local",
     "score": 16, "source": "tests/test_python.py:96"},
    # A table of the caller's (tests/test_python.py:100-101).
    {"kind": "score", "reference": "ACGTAC", "query": "ACGTAC", "scoring": TABULATED, "mode": "global", "score": 30,
     "source": "tests/test_python.py:100-101"},
    # Gap-affine (4,6,2) as a Scoring: Costs.affine(4,6,2)'s distance 12 is score -12
    # (tests/test_python.py:78; scoring.mojo:202-215; benchmarks/batches.mojo:18-21 maps costs to scores).
    {"kind": "score", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "scoring": CONFIG2, "mode": "global",
     "score": -12, "source": "tests/test_python.py:78 (score -12 under Costs.affine(4,6,2))"},
    # Unit-cost distances (tests/test_alignment.mojo:343-361; tests/test_python.py:5-6, 67).
    {"kind": "distance", "reference": "ACGT", "query": "ACGT", "distance": 0, "source": "tests/test_alignment.mojo:349"},
    {"kind": "distance", "reference": "ACGT", "query": "AGT", "distance": 1, "source": "tests/test_alignment.mojo:350"},
    {"kind": "distance", "reference": "ACGT", "query": "", "distance": 4, "source": "tests/test_alignment.mojo:351"},
    {"kind": "distance", "reference": "", "query": "ACG", "distance": 3, "source": "tests/test_alignment.mojo:352"},
    {"kind": "distance", "reference": "AAAA", "query": "TTTT", "distance": 4, "source": "tests/test_alignment.mojo:353"},
    {"kind": "distance", "reference": "ACGTACGT", "query": "TACGTACG", "distance": 2,
     "source": "tests/test_alignment.mojo:354-355"},
    {"kind": "distance", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "distance": 2,
     "source": "tests/test_python.py:67; python/dinara_align/__init__.py:7-8"},
]

# Alignments under Costs, the CIGAR the Ties rule names. `costs` is dinara_costs' nine fields in order;
# `cost` None means past `max_cost`.
UNIT = [1, 0, 1, -1, 0, 0, 0, -1, 0]
AFFINE = [4, 6, 2, -1, 0, 0, 0, -1, 0]
DEAR_DELETIONS = [4, 6, 2, -1, 0, 20, 5, -1, 0]
KNOWN += [
    {"kind": "costs", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "costs": UNIT, "ties": "left",
     "eqx": True, "cost": 2, "cigar": "4=1D2=1I6=", "source": "tests/test_python.py:71-72"},
    {"kind": "costs", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "costs": UNIT, "ties": "left",
     "eqx": False, "cost": 2, "cigar": "4M1D2M1I6M", "source": "tests/test_python.py:73"},
    {"kind": "costs", "reference": "ACGTTTTACG", "query": "ACGTTTACG", "costs": AFFINE, "ties": "left", "eqx": True,
     "cost": 8, "cigar": "3=1D6=", "source": "tests/test_python.py:74; tests/test_alignment.mojo:2162"},
    {"kind": "costs", "reference": "ACGTTTTACG", "query": "ACGTTTACG", "costs": AFFINE, "ties": "right",
     "eqx": True, "cost": 8, "cigar": "6=1D3=", "source": "tests/test_python.py:75; tests/test_alignment.mojo:2163"},
    {"kind": "costs", "reference": "ACGTTTTACG", "query": "ACGTTTACG", "costs": UNIT, "ties": "left", "eqx": True,
     "cost": 1, "cigar": "3=1D6=", "source": "tests/test_alignment.mojo:2199"},
    {"kind": "costs", "reference": "ACGTTTTACG", "query": "ACGTTTACG", "costs": UNIT, "ties": "right", "eqx": True,
     "cost": 1, "cigar": "6=1D3=", "source": "tests/test_alignment.mojo:2222"},
    {"kind": "costs", "reference": "ACGT", "query": "ACGT", "costs": UNIT, "ties": "left", "eqx": True, "cost": 0,
     "cigar": "4=", "source": "tests/test_python.py:76"},
    {"kind": "costs", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "costs": AFFINE, "ties": "left",
     "eqx": True, "max_cost": 11, "cost": None, "source": "tests/test_python.py:78"},
    {"kind": "costs", "reference": "ACGTACGTTTGCA", "query": "ACGTCGTTTTGCA", "costs": AFFINE, "ties": "left",
     "eqx": True, "max_cost": 12, "cost": 12, "cigar": "4=3X6=", "source": "tests/test_python.py:79, 81"},
    {"kind": "costs", "reference": "ACGACGT", "query": "ACGTACGT", "costs": DEAR_DELETIONS, "ties": "left",
     "eqx": True, "cost": 8, "source": "tests/test_python.py:85"},
    {"kind": "costs", "reference": "ACGTACGT", "query": "ACGACGT", "costs": DEAR_DELETIONS, "ties": "left",
     "eqx": True, "cost": 25, "source": "tests/test_python.py:86"},
]


def mutated(text: str, rate: float, rng: random.Random) -> str:
    """About `rate` of the letters substituted, deleted or followed by an inserted letter, a third each
    (the rule of the reference's tests/test_python.py:26-43)."""
    out = []
    for letter in text:
        roll = rng.random()
        if roll < rate / 3:
            out.append(rng.choice("ACGT"))
        elif roll < 2 * rate / 3:
            continue
        elif roll < rate:
            out.append(letter + rng.choice("ACGT"))
        else:
            out.append(letter)
    return "".join(out)


def dp_distance(a: str, b: str) -> int:
    """The edit distance by the full matrix a row at a time (tests/test_python.py:16-23's check)."""
    row = list(range(len(b) + 1))
    for i, x in enumerate(a, 1):
        previous, row[0] = row[0], i
        for j, y in enumerate(b, 1):
            previous, row[j] = row[j], min(row[j] + 1, row[j - 1] + 1, previous + (x != y))
    return row[-1]


def gaps(scoring: dict) -> tuple:
    return oracle.kernel_gaps(scoring["opening"], scoring["extension"])


def main() -> None:
    with open(os.path.join(HERE, "known_answers.json"), "w") as out:
        json.dump(KNOWN, out, indent=1)
    rng = random.Random(7)
    pairs = []
    for trial in range(200):
        reference = "".join(rng.choice("ACGT") for _ in range(rng.randrange(0, 120)))
        query = mutated(reference, [0.0, 0.05, 0.2, 0.5][trial % 4], rng)
        entry = {"reference": reference, "query": query, "distance": dp_distance(reference, query)}
        for name, scoring in (("dna", DNA), ("config2", CONFIG2)):
            table = scoring["table"]
            op, ex = gaps(scoring)
            a, b = oracle.codes(reference), oracle.codes(query)
            score, cigar, _, _ = oracle.gotoh_align(a, b, table, 4, op, ex, oracle.GLOBAL)
            local, local_cigar, top, bottom = oracle.gotoh_align(a, b, table, 4, op, ex, oracle.LOCAL)
            entry[name] = {"global": score, "global_cigar": cigar, "local": local, "local_cigar": local_cigar}
        pairs.append(entry)
    with open(os.path.join(HERE, "random_pairs.json"), "w") as out:
        json.dump({"generator": "random.Random(7), tests/test_python.py:120-128 rules", "pairs": pairs}, out)


if __name__ == "__main__":
    main()
