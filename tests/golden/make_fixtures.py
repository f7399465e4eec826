"""Regenerate the committed fixtures under tests/golden/.

Run where a reference tree is mounted, giving its root:

    python tests/golden/make_fixtures.py <reference tree>

* models/*.json: the reference's earth-model input files used by the
  configurations and by the reference's own model-reader known-answer test
  (f90/testReadNodeEarthmodel.f90).  They are input data, copied verbatim so
  the GPU tests and the bench can run where the reference is absent.
* oracle_fk_global_small.npz: the CPU oracle's FK spectra (complex128, as
  (frequency index, degree index, node, spectrum)) of frequencies 8 and 30 of
  the global configuration.  Regression vectors: they pin the oracle and the
  GPU parity form against later changes (made with --oracle; no reference tree
  needed).
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = ["prem-no-ocean_si.json", "ak135q.json"]


def oracle_vectors():
    sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
    sys.path.insert(0, os.path.join(HERE, "..", ".."))
    import numpy as np
    import oracle
    from gemini_unified_b200 import configs, model as M
    w = configs.WORKLOADS["global_small"]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    o = oracle.Oracle(m, ex)
    pc = M.fk_params_c(w.params, jre)
    out = {}
    for jf in (8, 30):
        n = int(g.nwn[jf - 1])
        spec, status, _ = o.fk_frequency(pc, jf, n, M.nsp_for(w.params))
        out["jf%d" % jf] = spec
        out["status%d" % jf] = status
    np.savez_compressed(os.path.join(HERE, "oracle_fk_global_small.npz"), **out)
    print("wrote oracle_fk_global_small.npz")


def main(ref):
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    for m in MODELS:
        shutil.copyfile(os.path.join(ref, "earthmodels", m), os.path.join(HERE, "models", m))
        print("wrote", m)


if __name__ == "__main__":
    if "--oracle" in sys.argv:
        oracle_vectors()
    elif len(sys.argv) == 2:
        main(sys.argv[1])
    else:
        sys.exit("usage: make_fixtures.py <reference tree> | --oracle")
