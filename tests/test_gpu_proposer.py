"""Learned step/order proposer: training kernels against the FP64 restatement,
and what the trained network (weights trained on the global configuration by
python -m gemini_unified_b200.proposer) changes in the solver.

The proposer only chooses each lane's order target and initial steps; the
error control still accepts or rejects every step, so the spectra change at
the level of the integrator's own tolerance.  The bar is the seismogram bar:
1e-5 relative L2 over all traces against the plain FP64 reference form (the
reference's own integration error at eps = 1e-5, measured against eps = 1e-8,
is 9e-6 on the same measure)."""
import numpy as np
import pytest

from gemini_unified_b200 import configs, model as M

pytestmark = pytest.mark.gpu


def test_gradient_matches_fp64_restatement(gpu):
    import proposer_mlp
    from gemini_unified_b200 import proposer
    rng = np.random.default_rng(3)
    w = proposer.init_weights(1) + rng.normal(0, 0.05, proposer.NPARAM).astype(np.float32)
    x = rng.normal(0, 1, (300, 11)).astype(np.float32)
    y = rng.normal(0, 0.3, (300, 3)).astype(np.float32)
    mask = (rng.random((300, 3)) > 0.2).astype(np.float32)
    loss, grad = proposer.gradient(w, x, y, mask)
    loss64, grad64 = proposer_mlp.loss_and_grad(w, x, y, mask)
    assert abs(loss - loss64) <= 1e-5 * loss64
    assert np.abs(grad - grad64).max() <= 1e-5 * np.abs(grad64).max()


def test_training_kernels_fit_a_known_function(gpu):
    from gemini_unified_b200 import proposer
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (8192, 11)).astype(np.float32)
    y = np.stack([np.sin(x[:, 0]) + 0.3 * x[:, 1] ** 2, np.tanh(x[:, 2] - x[:, 3]), 0.5 * x[:, 4] * x[:, 5]], 1)
    mask = np.ones_like(y, np.float32)
    w, norm, hist = proposer.train(x, y.astype(np.float32), mask, epochs=60, batch=1024, lr=3e-3)
    assert np.all(np.isfinite(hist)) and hist[-1] < 0.1 * hist[0]
    # the FP64 restatement agrees with the trained network's loss
    import proposer_mlp
    xs = (x - norm[:11]) / norm[11:]
    out, _, _ = proposer_mlp.forward(w, xs)
    assert float(((out - y) ** 2).mean()) < 0.1 * hist[0]


def test_trained_proposer_on_the_global_configuration(gpu):
    """The committed network against the solver without it: fewer extrapolation
    attempts (lane-level work), all items converge, seismograms within 1e-5."""
    from gemini_unified_b200 import proposer
    from gemini_unified_b200.fk import GeminiFK, synth_params
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    runs = {}
    for name, backend, use in (("plain", 1, 0), ("fast", 2, 0), ("fast+proposer", 2, proposer.USE_ORDER)):
        fk = GeminiFK(m, ex, backend=backend)
        if use:
            proposer.enable(fk, proposer.WEIGHTS, use, 0.1)
        gre, gim, _, st = fk.run(w.params, jre, g.nf1, g.nf2, f64=False)
        assert np.all(st == 0)
        runs[name] = (gre, gim, fk.stats())
    a_fast, a_prop = runs["fast"][2]["attempts"], runs["fast+proposer"][2]["attempts"]
    print("attempts fast %d, with proposer %d (%.4f)" % (a_fast, a_prop, a_prop / a_fast))
    assert a_prop < a_fast
    src = ex.node_index(m.rearth - 10000.0)
    theta, phi, propdir = w.stations()
    mt = configs.unit_moment_tensors()
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    syn = GeminiFK(m, ex)
    tr = {k: syn.synthetics(sp, g.nwn, v[0][src - 1], v[1][src - 1], theta, phi, propdir, mt).astype(np.float64)
          for k, v in runs.items()}
    err = np.linalg.norm(tr["fast+proposer"] - tr["plain"]) / np.linalg.norm(tr["plain"])
    print("seismogram relative L2 over all traces vs the plain form: %.2e" % err)
    assert err <= 1e-5
