"""Many independent reconstructions in one call (fpm_solve_batch) and the epoch graphs.

fpm_solve_batch runs every instance on a worker context of its own, concurrently over a
pool of streams, each instance's epochs after the first replayed from a captured CUDA
graph.  Neither changes an instance's arithmetic, so every result must equal the one a
separate fpm_solve gives, bit for bit: the object, pupil, spectrum and per-epoch loss.
Instances mix the fused power-of-two pipeline and the any-size path, uint16 and float
stacks, both losses and uneven LED counts and batch sizes.
"""
import os

import numpy as np
import pytest

from conftest import led_matlab, to_matlab_stack, dataset

pytestmark = pytest.mark.gpu


def _instances():
    out = []
    specs = [(32, 4, 3, 8, "anisotropic", True), (48, 4, 5, 8, "isotropic", False),
             (64, 2, 5, 13, "anisotropic", True), (40, 5, 3, 4, "anisotropic", False),
             (64, 3, 5, 26, "isotropic", True), (128, 4, 5, 8, "anisotropic", True)]
    for k, (h, p, grid, B, loss, raw) in enumerate(specs):
        ds = dataset(h, p, grid, seed=20 + k, aberration=True)
        L = len(ds.led_idx) - k % 3        # uneven LED counts
        Y = ds.raw[:L] if raw else ds.Y[:L]
        out.append(dict(O0=ds.O0, P0c=ds.P0c, Y=to_matlab_stack(Y), led_idx=led_matlab(ds.led_idx[:L]),
                        P0=ds.pupil0, pratio=p, epochs=3, batch=B, lr=1e-3, loss=loss))
    return out


@pytest.mark.parametrize("eager", [False, True])
def test_solve_batch_equals_separate_solves(engine, eager):
    inst = _instances()
    res, st = engine.solve_batch(inst, eager=eager, spectrum=True)
    assert st == [0] * len(inst)
    for a, r in zip(inst, res):
        one = engine.solve(a["O0"], a["P0c"], a["Y"], a["led_idx"], a["P0"], a["pratio"],
                           a["epochs"], a["batch"], lr=a["lr"], loss=a["loss"])
        for k in ("object", "pupil", "spectrum", "loss"):
            np.testing.assert_array_equal(np.asarray(r[k]), np.asarray(one[k]), err_msg=k)


def test_solve_batch_reports_each_instance(engine):
    """A bad instance fails alone with its own status; the others still solve."""
    inst = _instances()[:3]
    bad = dict(inst[1])
    bad["led_idx"] = np.full_like(inst[1]["led_idx"], 10 ** 6)      # corners outside [1, H]
    res, st = engine.solve_batch([inst[0], bad, inst[2]])
    assert st[0] == 0 and st[2] == 0 and st[1] == 1
    assert "instance 1" in engine.lib.fpm_last_error(engine._ctx).decode()
    one = engine.solve(inst[2]["O0"], inst[2]["P0c"], inst[2]["Y"], inst[2]["led_idx"],
                       inst[2]["P0"], inst[2]["pratio"], inst[2]["epochs"], inst[2]["batch"],
                       lr=inst[2]["lr"], loss=inst[2]["loss"])
    np.testing.assert_array_equal(np.asarray(res[2]["object"]), np.asarray(one["object"]))


@pytest.mark.parametrize("h,p", [(64, 4), (48, 4)])
def test_epoch_graphs_equal_eager_epochs(engine, h, p):
    """fpm_solve replays epochs 2.. from a captured graph; FPM_GRAPHS=0 launches every
    kernel instead.  Both must agree bit for bit, across a learning-rate change (one graph
    per learning rate: lr_halve_after = 1 over 4 epochs)."""
    ds = dataset(h, p, 5, seed=4, aberration=True)
    args = (ds.O0, ds.P0c, to_matlab_stack(ds.raw), led_matlab(ds.led_idx), ds.pupil0, p, 4, 8)
    runs = {}
    for flag in ("1", "0"):
        os.environ["FPM_GRAPHS"] = flag
        try:
            runs[flag] = engine.solve(*args, lr=1e-3, lr_halve_after=1)
        finally:
            del os.environ["FPM_GRAPHS"]
    for k in ("object", "pupil", "spectrum", "loss"):
        np.testing.assert_array_equal(np.asarray(runs["1"][k]), np.asarray(runs["0"][k]), err_msg=k)


def test_kept_epoch_graph_equals_a_fresh_one():
    """A context keeps its executable epoch graph between solves: a later capture with the
    same nodes (another learning rate, another problem of the same plan) writes its
    parameters into it, one with other nodes replaces it.  Every solve of a context that
    went through both must equal, bit for bit, the same solve in a fresh context
    (problems A and B of one shape, then C of another; lr halved after epoch 1, so each
    solve also captures twice)."""
    import fpm_b200
    probs = []
    for seed, h, p in ((31, 64, 4), (32, 64, 4), (33, 48, 4), (34, 64, 4)):
        ds = dataset(h, p, 5, seed=seed, aberration=True)
        probs.append((ds.O0, ds.P0c, to_matlab_stack(ds.raw), led_matlab(ds.led_idx),
                      ds.pupil0, p, 4, 8))
    with fpm_b200.Engine(0) as kept:
        for args in probs:
            a = kept.solve(*args, lr=1e-3, lr_halve_after=1)
            with fpm_b200.Engine(0) as fresh:
                b = fresh.solve(*args, lr=1e-3, lr_halve_after=1)
            for k in ("object", "pupil", "spectrum", "loss"):
                np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)
