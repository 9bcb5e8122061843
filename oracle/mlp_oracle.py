"""CPU oracle of the learned band predictor: its 4-mer sketch and its network's forward and backward pass in
float64 numpy.

TEST INFRASTRUCTURE ONLY: the tests check the GPU's features and training gradients against these; nothing
in the product imports it. The layout follows the library's flat parameter vector: w1 [258][64], b1 [64],
w2 [64][64], b2 [64], w3 [64], b3.
"""

from __future__ import annotations

import numpy as np

INPUTS, HIDDEN = 258, 64
SIZES = [("w1", (INPUTS, HIDDEN)), ("b1", (HIDDEN,)), ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)), ("w3", (HIDDEN,)),
         ("b3", (1,))]
PARAMETERS = sum(int(np.prod(shape)) for _, shape in SIZES)
CODES = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3}


def unpack(flat: np.ndarray) -> dict:
    out, at = {}, 0
    for name, shape in SIZES:
        size = int(np.prod(shape))
        out[name] = np.asarray(flat[at:at + size], dtype=np.float64).reshape(shape)
        at += size
    return out


def pack(parts: dict) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], dtype=np.float64).ravel() for name, _ in SIZES])


def kmer_counts(sequence: bytes, k: int = 4) -> np.ndarray:
    """Counts of each k-mer (A=0, C=1, G=2, T=3, first letter most significant); a k-mer holding another
    letter is skipped."""
    counts = np.zeros(4 ** k, dtype=np.int64)
    for start in range(len(sequence) - k + 1):
        code = 0
        for letter in sequence[start:start + k]:
            value = CODES.get(letter)
            if value is None:
                code = -1
                break
            code = code * 4 + value
        if code >= 0:
            counts[code] += 1
    return counts


def features(reference: bytes, query: bytes) -> np.ndarray:
    """The 258 inputs: each 4-mer count difference squared, times 32 over the mean length; the length
    ratio; and the 6-mer count differences' squares summed, over the mean length."""
    out = np.zeros(INPUTS, dtype=np.float64)
    mean = 0.5 * (len(reference) + len(query))
    difference = (kmer_counts(reference) - kmer_counts(query)).astype(np.float64)
    out[:256] = 32.0 * difference ** 2 / max(mean, 1.0)
    low, high = min(len(reference), len(query)), max(len(reference), len(query))
    out[256] = low / high if high > 0 else 1.0
    sixes = (kmer_counts(reference, 6) - kmer_counts(query, 6)).astype(np.float64)
    out[257] = float((sixes ** 2).sum()) / max(mean, 1.0)
    return out


def forward(parts: dict, x: np.ndarray) -> tuple:
    """x: [batch, 258]; returns (y [batch], cache)."""
    z1 = x @ parts["w1"] + parts["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ parts["w2"] + parts["b2"]
    h2 = np.maximum(z2, 0.0)
    y = h2 @ parts["w3"] + parts["b3"][0]
    return y, (x, z1, h1, z2, h2)


def gradients(flat: np.ndarray, x: np.ndarray, targets: np.ndarray) -> tuple:
    """The mean squared error's gradient (flat) and the mean squared error."""
    parts = unpack(flat)
    y, (x, z1, h1, z2, h2) = forward(parts, x)
    batch = len(targets)
    dy = 2.0 * (y - targets) / batch
    grads = {"w3": h2.T @ dy, "b3": np.array([dy.sum()])}
    dz2 = np.outer(dy, parts["w3"]) * (z2 > 0)
    grads["w2"] = h1.T @ dz2
    grads["b2"] = dz2.sum(axis=0)
    dz1 = (dz2 @ parts["w2"].T) * (z1 > 0)
    grads["w1"] = x.T @ dz1
    grads["b1"] = dz1.sum(axis=0)
    return pack(grads), float(np.mean((y - targets) ** 2))
