"""The FK-spectra file (HDF5, the reference's layout) between the GPU's FK
spectra and its seismograms: spectra of the global configuration computed on
the GPU are written frequency slab by frequency slab, read back, and the
seismograms computed from the file's node spectra and frequency grid equal the
seismograms from the spectra in memory bit for bit."""
import numpy as np
import pytest

from gemini_unified_b200 import configs, fkfile, model as M

pytestmark = pytest.mark.gpu


def test_seismograms_from_the_fk_file_equal_the_direct_path(gpu, tmp_path):
    from gemini_unified_b200.fk import GEM_BACKEND_GPU_FAST, GeminiFK, synth_params
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    fk = GeminiFK(m, ex, backend=GEM_BACKEND_GPU_FAST)
    path = str(tmp_path / "gfk.MOMENT")
    parts = []
    with fkfile.FKFileWriter(path, m, ex, w.params, jre, earth_model_name=m.name) as fw:
        for a, b in ((27, g.nf2), (g.nf1, 26)):
            gre, gim, _, st = fk.run(w.params, jre, a, b, f64=False)
            assert np.all(st == 0)
            fw.write_slab(a, b, gre, gim)
            parts.append((a, gre, gim))
    parts.sort(key=lambda p: p[0])
    gre = np.concatenate([p[1] for p in parts], axis=2)
    gim = np.concatenate([p[2] for p in parts], axis=2)
    src = ex.node_index(m.rearth - 10000.0)
    theta, phi, propdir = w.stations()
    mt = configs.unit_moment_tensors()
    sp = synth_params(g, 10, w.nsamp, w.dt, w.filspecs)
    direct = fk.synthetics(sp, g.nwn, gre[src - 1], gim[src - 1], theta, phi, propdir, mt)
    with fkfile.FKFile(path) as f:
        gf = f.grid()
        fr, fi = f.read_node(src)
        assert np.array_equal(fr.view(np.uint32), gre[src - 1].view(np.uint32))
        assert np.array_equal(fi.view(np.uint32), gim[src - 1].view(np.uint32))
        spf = synth_params(gf, f.meta.nsp, w.nsamp, w.dt, w.filspecs)
        assert (spf.df, spf.sigma, spf.nf1, spf.nf2) == (sp.df, sp.sigma, sp.nf1, sp.nf2)
        fromfile = fk.synthetics(spf, gf.nwn, fr, fi, theta, phi, propdir, mt)
    assert np.array_equal(fromfile.view(np.uint32), direct.view(np.uint32))
