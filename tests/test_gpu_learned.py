"""The learned band on the GPU: its sketch and its training gradients against the CPU oracle
(oracle/mlp_oracle.py), distances exact under it, and what it gains over plain band doubling."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def learned(da):
    from dinara_align import learned as module

    return module


def test_features_match_oracle(da, learned):
    import mlp_oracle

    rng = np.random.default_rng(3)
    refs, queries = [], []
    for _ in range(40):
        n = int(rng.integers(0, 700))
        a = "".join(rng.choice(list("ACGT"), size=n))
        b = "".join(ch if rng.random() > 0.1 else rng.choice(list("ACGTN")) for ch in a)
        refs.append(a)
        queries.append(b)
    refs.append("AC")
    queries.append("")
    tape = da.Tape.of(refs, queries)
    got = learned.Predictor().features(tape)
    expected = np.stack([mlp_oracle.features(r.encode(), q.encode()) for r, q in zip(refs, queries)])
    np.testing.assert_allclose(got, expected, rtol=1e-5, atol=1e-6)


def test_gradients_match_oracle(learned):
    """The training kernels' gradients (tiled products forward and back) against float64 numpy."""
    import mlp_oracle

    rng = np.random.default_rng(4)
    flat = rng.normal(0, 0.1, size=learned.PARAMETERS).astype(np.float32)
    x = rng.normal(0, 0.5, size=(300, 258)).astype(np.float32)
    t = rng.uniform(0, 0.2, size=300).astype(np.float32)
    predictor = learned.Predictor()
    predictor.install(flat, 1.0, 0.0)
    got, loss = predictor.gradients(x, t)
    expected, expected_loss = mlp_oracle.gradients(flat.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    # fp32 sums in another order: within 1e-3 of the largest gradient, and the loss to 1e-5 relative.
    scale = np.abs(expected).max()
    np.testing.assert_allclose(got, expected, rtol=1e-3, atol=1e-3 * scale)
    assert abs(loss - expected_loss) <= 1e-5 * max(1.0, expected_loss)


def test_learned_band_is_exact_and_gains(da, oracle, learned, tmp_path):
    """A predictor trained on the GPU starts each pair near its distance: every distance stays exact (the
    doubling that follows is plain band doubling's), and the band sweeps fewer words than plain doubling's
    default start."""
    from dinara_align import workloads

    predictor = learned.Predictor()
    report = predictor.train(pairs=100_000, length=(100, 5000), epochs=4, batch=1024, seed=11)
    # Better than the error rates' own spread (a rate uniform in 0.5-15% has a variance near 0.0017).
    assert report["steps"] > 0 and report["validation_loss"] < 0.001, report
    tape = workloads.uneven_unit_cost(800, high=5000, seed=19)
    expected = oracle.batch_distances(tape.letters[: tape.offsets[-1]], tape.offsets, start=-1, threads=8)
    plain, plain_report = da.distances_tape(tape, report=True)
    learned_found, learned_report = da.distances_tape(tape, policy=da._native.BAND_LEARNED, report=True)
    np.testing.assert_array_equal(plain, expected)
    np.testing.assert_array_equal(learned_found, expected)
    assert learned_report["words_swept"] < 0.8 * plain_report["words_swept"], (plain_report, learned_report)
    # A batch of several units streams its letters, each unit predicted and doubled on its own lane with
    # the context's predictor: the same distances.
    big = workloads.uneven_unit_cost(70_000, high=600, seed=23)
    expected_big = oracle.batch_distances(big.letters[: big.offsets[-1]], big.offsets, start=-1, threads=8)
    np.testing.assert_array_equal(da.distances_tape(big, policy=da._native.BAND_LEARNED), expected_big)
    predicted, thresholds = predictor.predict(tape)
    assert (thresholds >= 1).all() and np.isfinite(predicted).all()
    # The blob keeps every length class's margin: loaded back, the thresholds are the same.
    margins = predictor.margins()
    blob = str(tmp_path / "predictor.npz")
    predictor.save(blob)
    predictor.install(np.zeros(learned.PARAMETERS, dtype=np.float32), 1.0, 0.0)
    predictor.load(blob)
    assert predictor.margins() == margins
    np.testing.assert_array_equal(predictor.predict(tape)[1], thresholds)
