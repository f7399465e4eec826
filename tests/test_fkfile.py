"""The FK-spectra file (HDF5 layout of computeGreenFKSpectraForSynthetics) on the CPU.

* The HDF5 reader parses a file written by the HDF5 library itself: a
  MATLAB 7.3 test file that SciPy ships (superblock after a 512-byte user
  block, group B-tree, symbol-table node, local heap, version-1 object
  headers, a float64 contiguous dataset, a string attribute).  Skipped where
  SciPy's test data are not installed.
* Files from the writer follow the structures of the HDF5 format
  specification that the library reads (checked byte by byte), and read back
  through the same reader.
* An FK-spectra file written slab by slab, out of order, reads back with the
  reference's metadata and every node's spectra bit for bit.
* The node properties stored with the file agree with an independent natural
  cubic spline of the model (SciPy).
"""
import dataclasses
import os
import struct

import numpy as np
import pytest

from gemini_unified_b200 import configs, fkfile, h5file, model as M

MAT73 = None
try:
    import scipy.io
    MAT73 = os.path.join(os.path.dirname(scipy.io.__file__), "matlab", "tests", "data", "testhdf5_7.4_GLNX86.mat")
except ImportError:
    pass


@pytest.mark.skipif(MAT73 is None or not os.path.exists(MAT73), reason="SciPy's HDF5 test file is not installed")
def test_reader_parses_a_file_written_by_the_hdf5_library():
    with h5file.H5Reader(MAT73) as r:
        assert r.base == 512
        assert r.keys() == ["testdouble"]
        d = r["testdouble"]
        assert d.shape == (9, 1) and d.dtype == np.dtype("<f8")
        assert bytes(d.attrs["MATLAB_class"].item()) == b"double"
        np.testing.assert_allclose(d.read()[:, 0], np.pi / 4 * np.arange(9), rtol=0, atol=1e-15)


def test_writer_structures_follow_the_format_specification(tmp_path):
    p = str(tmp_path / "t.h5")
    w = h5file.H5Writer(p)
    w.set_attr("/", "identity", "Thu Dec  4 05:00:00 2026")
    w.set_attr("/", "ints", np.array([1, -2, 3], np.int32))
    w.create_group("grp")
    names = ["d%02d" % i for i in range(40)]        # two symbol-table nodes of up to 32 entries
    for i, n in enumerate(names):
        w.create_dataset("grp/" + n, np.full(3, i, np.float32))
    w.create_string("s", "ATTENUATION_AND_DISPERSION")
    w.create_dataset("big", shape=(2, 3, 5), dtype="<f4")
    w.close()
    b = open(p, "rb").read()
    # superblock version 0: 8-byte sizes, K 16/16, base 0, end-of-file address = file size
    assert b[:8] == h5file.SIGNATURE and b[8:13] == bytes(5) and b[13:15] == b"\x08\x08"
    assert struct.unpack_from("<HH", b, 16) == (h5file.LEAF_K, h5file.INTERNAL_K)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert (base, free, eof, drv) == (0, h5file.UNDEF, len(b), h5file.UNDEF)
    _, root, cache, _, tree, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert cache == 1
    # local heap: version 0, free list 'none' (1), the data segment starts with the empty name
    assert b[heap:heap + 5] == b"HEAP\x00"
    seg_size, free_head, seg = struct.unpack_from("<QQQ", b, heap + 8)
    assert free_head == h5file.HEAP_FREE_NULL and b[seg:seg + 8] == bytes(8) and seg_size % 8 == 0
    # group B-tree node: type 0, leaf level, key 0 = the empty name, room for 2K children
    assert b[tree:tree + 6] == b"TREE\x00\x00"
    assert struct.unpack_from("<Q", b, tree + 24)[0] == 0
    # object header version 1: messages start 16 bytes in, sizes are multiples of 8
    ver, _, nmsg, refc, size = struct.unpack_from("<BBHII", b, root)
    assert (ver, refc) == (1, 1) and size % 8 == 0
    p_ = root + 16
    for _ in range(nmsg):
        t, sz = struct.unpack_from("<HH", b, p_)
        assert sz % 8 == 0
        p_ += 8 + sz
    assert p_ == root + 16 + size
    with h5file.H5Reader(p) as r:
        assert sorted(r.keys()) == ["big", "grp", "s"]
        assert r.attrs["identity"].item() == b"Thu Dec  4 05:00:00 2026"
        assert r.attrs["ints"].tolist() == [1, -2, 3]
        g = r["grp"]
        assert g.keys() == names
        for i, n in enumerate(names):
            assert g[n].read().tolist() == [i, i, i]
        assert r["s"].read().item() == b"ATTENUATION_AND_DISPERSION"
        assert r["big"].shape == (2, 3, 5) and not r["big"].read().any()


def _write_case(path, params, slabs, seed=3):
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(params, m.rearth)
    nsp = M.nsp_for(params)
    rng = np.random.default_rng(seed)
    full = (rng.standard_normal((2, ex.nnod, nsp, int(g.nkfmax))) * 1e-9).astype(np.float32)
    full[:, :, 2:4, 0] = np.nan    # the l = 0 V components of the first frequency
    koff = np.concatenate([[0], np.cumsum(g.nwn[g.nf1 - 1: g.nf2])])
    fw = fkfile.FKFileWriter(path, m, ex, params, jre, earth_model_name="prem-no-ocean_si.json",
                             identity="Thu Dec  4 05:00:00 2026")
    for a, b in slabs:
        k0, k1 = koff[a - g.nf1], koff[b - g.nf1 + 1]
        fw.write_slab(a, b, full[0][:, :, k0:k1], full[1][:, :, k0:k1])
    fw.close()
    return m, ex, jre, g, nsp, full


@pytest.mark.parametrize("source", ["MOMENT", "FORCE"])
def test_fk_file_round_trip_slab_by_slab(tmp_path, source):
    w = configs.WORKLOADS["global_small"]
    params = dataclasses.replace(w.params, source_type=source)
    g = M.frequency_grid(params, w.model().rearth)
    slabs = [(30, g.nf2), (g.nf1, 9), (10, 29)]       # out of order, as ranks deliver them
    path = str(tmp_path / "gfk.MOMENT")
    m, ex, jre, g, nsp, full = _write_case(path, params, slabs)
    with fkfile.FKFile(path) as f:
        mt = f.meta
        assert mt.identity == "Thu Dec  4 05:00:00 2026"
        assert mt.earth_model_name == "prem-no-ocean_si.json" and mt.attenuation_mode == params.attmode
        f32 = lambda v: float(np.float32(v))
        assert (mt.rearth, mt.re, mt.sigma, mt.df, mt.dwn, mt.fref) == (
            f32(m.rearth), f32(ex.r[jre - 1]), f32(g.sigma), f32(g.df), f32(g.dwn), f32(m.fref))
        assert (mt.nf1, mt.nf2, mt.nkfmax, mt.nwnmax, mt.dsvstep, mt.derivflag, mt.numtasks, mt.global_) == (
            g.nf1, g.nf2, int(g.nkfmax), g.nwnmax, 2, 0, 1, 1)
        assert np.array_equal(mt.nwn, g.nwn[: g.nf2])
        istyp = 1 if source == "MOMENT" else 0
        assert (mt.istyp, mt.ncsph, mt.nctor, mt.njsph, mt.njtor) == (istyp, 4, 2, 4 if istyp else 2, 2 if istyp else 1)
        assert mt.nsp == nsp and mt.nnod == ex.nnod
        # the reader's count of spectra (greenFKSpectra.f90:223-229) matches the file
        mask = mt.dsvmask()
        assert int(mask[:6].sum()) * mt.njsph + int(mask[6:].sum()) * mt.njtor == nsp
        # spectrum positions: W of the first toroidal jump follows the spheroidal ones
        assert mt.position(7, 1) == 2 * mt.njsph + 1
        assert np.array_equal(mt.node_radii, np.asarray(ex.r, np.float32))
        for jr in range(1, ex.nnod + 1):
            re, im = f.read_node(jr)
            assert np.array_equal(re.view(np.uint32), full[0][jr - 1].view(np.uint32))
            assert np.array_equal(im.view(np.uint32), full[1][jr - 1].view(np.uint32))


def test_fk_file_rejects_a_slab_of_the_wrong_shape(tmp_path):
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    fw = fkfile.FKFileWriter(str(tmp_path / "x"), m, ex, w.params, ex.node_index(w.rec_radius))
    with pytest.raises(ValueError):
        fw.write_slab(5, 6, np.zeros((ex.nnod, 10, 3), np.float32), np.zeros((ex.nnod, 10, 3), np.float32))
    with pytest.raises(ValueError):
        fw.write_slab(1, 2, np.zeros((1,)), np.zeros((1,)))
    fw.close()


def test_node_properties_follow_a_natural_cubic_spline_of_the_model():
    from scipy.interpolate import CubicSpline
    w = configs.WORKLOADS["batched_fk"]
    m = w.model()
    ex = w.nodes(m)
    ro, qinv, el = M.node_elastic_constants(m, ex)
    assert np.all(el.imag == 0)                       # ELASTIC mode
    rk = m.rk
    for i in range(ex.nnod):
        nl = int(ex.layer[i])
        top = int(m.iktop[nl - 1])
        bot = int(m.ikbot[nl - 1]) if nl > 1 else top
        if top - bot < 2:
            continue
        x = rk[bot - 1: top]
        cs = CubicSpline(x, m.ro[bot - 1: top], bc_type="natural")
        assert abs(cs(ex.r[i]) - ro[i]) <= 1e-10 * ro[i]
        mu = m.ro[bot - 1: top] * m.vsv[bot - 1: top] ** 2         # isotropic model: mu = rho vs^2
        assert abs(CubicSpline(x, mu, bc_type="natural")(ex.r[i]) - el[i, 6].real) <= 1e-9 * el[i, 6].real
        qm = 1.0 / m.qm[bot - 1: top]
        assert abs(CubicSpline(x, qm, bc_type="natural")(ex.r[i]) - qinv[i, 1]) <= 1e-12
