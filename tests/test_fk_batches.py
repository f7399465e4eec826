"""Batched FK run with a completion record (host logic, no GPU): a run stopped by a
failing batch resumes where it stopped, the resumed result equals an uninterrupted
run, and a folder of another run is refused."""
import dataclasses

import numpy as np
import pytest

from gemini_unified_b200 import configs, fk_batches, model as M


class FakeFK:
    """Stands in for GeminiFK: deterministic spectra per (jf, iwn), optional failure."""

    def __init__(self, m, ex, fail_at=None):
        self.model, self.nodes, self.fail_at, self.calls = m, ex, fail_at, []

    def run(self, params, jre, a, b, f32=True, f64=False, raise_on_failure=True):
        if self.fail_at is not None and a == self.fail_at:
            raise RuntimeError("injected failure in batch %d" % a)
        self.calls.append((a, b))
        g = M.frequency_grid(params, self.model.rearth)
        nkf = int(g.nwn[a - 1: b].sum())
        k = np.arange(nkf, dtype=np.float32) + float(g.nwn[: a - 1].sum())
        gre = np.broadcast_to(k, (self.nodes.nnod, 10, nkf)).astype(np.float32) * 1e-3
        return gre, -gre, None, np.zeros(nkf, np.int32)


@pytest.fixture()
def setup(tmp_path):
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    return w, m, ex, ex.node_index(w.rec_radius), str(tmp_path / "run")


def test_resume_after_a_failed_batch(setup, tmp_path):
    w, m, ex, jre, out = setup
    g = M.frequency_grid(w.params, m.rearth)
    bs = fk_batches.batches(g.nf1, g.nf2, 8)
    assert bs[0][0] == g.nf1 and bs[-1][1] == g.nf2 and all(b[0] == a[1] + 1 for a, b in zip(bs, bs[1:]))
    with pytest.raises(RuntimeError):
        fk_batches.run(FakeFK(m, ex, fail_at=bs[3][0]), w.params, jre, out, 8)
    first = fk_batches.load(out)
    assert first[0].shape[2] == sum(int(g.nwn[a - 1: b].sum()) for a, b in bs[:3])
    fk2 = FakeFK(m, ex)
    res = fk_batches.run(fk2, w.params, jre, out, 8)
    assert fk2.calls == bs[3:]                               # only the missing batches ran
    assert [c for _, c in res] == [False] * 3 + [True] * (len(bs) - 3)
    gre, gim, st = fk_batches.load(out)
    ref = str(tmp_path / "ref")
    fk_batches.run(FakeFK(m, ex), w.params, jre, ref, 8)
    r = fk_batches.load(ref)
    np.testing.assert_array_equal(gre, r[0])
    np.testing.assert_array_equal(gim, r[1])
    assert gre.shape == (ex.nnod, 10, int(g.nkfmax))
    fk3 = FakeFK(m, ex)
    fk_batches.run(fk3, w.params, jre, out, 8)
    assert fk3.calls == []                                   # everything recorded: nothing to do


def test_folder_of_another_run_is_refused(setup):
    w, m, ex, jre, out = setup
    fk_batches.run(FakeFK(m, ex), w.params, jre, out, 16)
    other = dataclasses.replace(w.params, eps=1e-6)
    with pytest.raises(ValueError):
        fk_batches.run(FakeFK(m, ex), other, jre, out, 16)


def test_export_to_the_fk_spectra_file(setup, tmp_path):
    """The recorded batches become one FK-spectra file in the reference's HDF5
    layout; a node read from it equals the batches' spectra of that node."""
    from gemini_unified_b200.fkfile import FKFile
    w, m, ex, jre, out = setup
    fk_batches.run(FakeFK(m, ex), w.params, jre, out, 16)
    path = str(tmp_path / "gfk.MOMENT")
    fk_batches.export(out, path, m, ex, w.params, jre)
    gre, gim, _ = fk_batches.load(out)
    with FKFile(path) as f:
        assert f.meta.nkfmax == gre.shape[2] and f.meta.nnod == ex.nnod
        for jr in (1, jre):
            re, im = f.read_node(jr)
            np.testing.assert_array_equal(re, gre[jr - 1])
            np.testing.assert_array_equal(im, gim[jr - 1])


def test_export_refuses_an_incomplete_run(setup, tmp_path):
    w, m, ex, jre, out = setup
    g = M.frequency_grid(w.params, m.rearth)
    with pytest.raises(RuntimeError):
        fk_batches.run(FakeFK(m, ex, fail_at=fk_batches.batches(g.nf1, g.nf2, 8)[2][0]), w.params, jre, out, 8)
    with pytest.raises(ValueError):
        fk_batches.export(out, str(tmp_path / "x"), m, ex, w.params, jre)
