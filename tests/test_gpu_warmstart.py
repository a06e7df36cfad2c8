"""What the learned warm start gains over N4 without it.

The shipped encoder (``n4b200/weights/warmstart_encoder.npy``, trained by
``python -m n4b200.warmstart train`` on 4096 GPU-generated 128x128x96
phantoms labelled by the plain GPU N4) is evaluated on held-out 256x256x176
phantoms (seeds disjoint from training and validation) against the same
batch run from zero lattices and against an untrained encoder.
"""
import pytest

pytestmark = pytest.mark.gpu


def test_trained_warm_start_saves_iterations(cuda):
    from n4b200.encoder import Encoder
    from n4b200.warmstart import evaluate, load_encoder
    r = evaluate(load_encoder(), n_eval=16, chunk=16)
    u = evaluate(Encoder(max_batch=64, seed=0), n_eval=16, chunk=16)
    print("trained", r)
    print("untrained", u)
    # the first-iteration rule keeps the prediction for (almost) every volume
    assert r["warm_kept"] >= 0.9
    # first level: the prediction is already near its converged lattice
    assert r["level1_iterations_warm"] <= 0.5 * r["level1_iterations_plain"]
    assert r["iterations_warm"] < r["iterations_plain"]
    # an untrained network of the same shape gains nothing
    assert r["iterations_warm"] < u["iterations_warm"]
    # same correction as without warm start, up to a global intensity scale
    assert r["max_abs_log_bias_diff_mask_mean_removed"] <= 0.01


def test_training_on_n4_labels_beats_the_mean_predictor(cuda):
    """A short run of the training pipeline (GPU phantoms -> plain N4 labels
    -> Adam on the tensor-core encoder) learns more than the label mean."""
    from n4b200.warmstart import train_encoder
    enc, rep = train_encoder(n_train=1024, n_val=128, shape=(64, 64, 48), epochs=10, batch=64, seed=11)
    print(rep)
    assert rep["loss_last_epoch"] < rep["loss_first_epoch"]
    assert rep["val_mse"] < 0.7 * rep["val_mse_of_mean_predictor"]
