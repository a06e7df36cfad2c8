"""What the learned warm start gains over N4 without it.

The shipped encoder (``n4b200/weights/warmstart_encoder.npy``, trained by
``python -m n4b200.warmstart train`` on 4096 GPU-generated 256x256x176
phantoms labelled by the plain GPU N4) is evaluated on held-out 256x256x176
phantoms (seeds disjoint from training and validation) against the same
batch run from zero lattices and against an untrained encoder.

The log-bias difference to the plain run is reported raw and with its mean
over the mask removed.  The residual N4 fits, logU - E(logU), does not change
when a constant is added to logU, so neither does any update or convergence
value: the constant of the log bias is never corrected, and whatever
constant the warm start hands over (plus the drift mean(residual) of every
iteration it runs) stays in the result.  The non-constant part is what N4
converges; it is held to 0.01.  The raw difference is measured and printed
(its distribution over 256 volumes is stated in the design notes); it is not
within 0.01.
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
    # the non-constant part of the correction agrees with the plain run's
    assert r["max_abs_log_bias_diff_mask_mean_removed"] <= 0.01
    # the raw difference (the constant mode): recorded, and kept from growing
    assert r["median_abs_log_bias_diff_mask"] <= 0.1


def test_training_on_n4_labels_beats_the_mean_predictor(cuda):
    """A short run of the training pipeline (GPU phantoms -> plain N4 labels
    one iteration before the first level stops -> Adam on the tensor-core
    encoder) learns more than the label mean."""
    from n4b200.warmstart import train_encoder
    enc, rep = train_encoder(n_train=1024, n_val=128, shape=(64, 64, 48), epochs=10, batch=64, seed=11)
    print(rep)
    assert rep["loss_last_epoch"] < rep["loss_first_epoch"]
    assert rep["val_mse"] < 0.7 * rep["val_mse_of_mean_predictor"]
