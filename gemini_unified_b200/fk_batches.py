"""FK spectra of a whole frequency band in batches, with a completion record for resume.

    python -m gemini_unified_b200.fk_batches --workload batched_fk --out runs/batched --batch 32 [--h5 gfk.MOMENT]

The reference writes each rank's frequency slab to the FK file as it completes it
(computeGreenFKSpectraForSynthetics.f90:508-519) and has no resume: a stopped run starts
again from FMIN.  Here each batch of frequencies is one GPU call; its float32 spectra and
per-item status go to ``spectra_<jf0>_<jf1>.npz`` in the output folder, and
``done.json`` lists the completed batches together with a fingerprint of the run's
parameters.  A second run with the same parameters skips the completed batches; a run
with other parameters refuses the folder.  Files are written to a temporary name and
renamed, so a batch that was interrupted is never recorded.  ``export`` writes the recorded
batches into one FK-spectra file in the reference's HDF5 layout (gemini_unified_b200.fkfile),
which the reference's computeSyntheticSeismograms reads.
"""
from __future__ import annotations

import argparse
import dataclasses
import hashlib
import json
import os
from typing import List, Sequence, Tuple

import numpy as np

from . import configs, model as M

RECORD = "done.json"


def batches(nf1: int, nf2: int, size: int) -> List[Tuple[int, int]]:
    """Consecutive frequency ranges jf0..jf1 of at most ``size`` frequencies covering nf1..nf2."""
    if size < 1:
        raise ValueError("batch size must be at least 1")
    return [(a, min(a + size - 1, nf2)) for a in range(nf1, nf2 + 1, size)]


def fingerprint(params: M.FKParams, jre: int, nodes_r: Sequence[float], extra: str = "") -> str:
    """Identity of a run: the FK parameters, the receiver node, the node radii."""
    h = hashlib.sha256()
    h.update(json.dumps(dataclasses.asdict(params), sort_keys=True, default=float).encode())
    h.update(str(int(jre)).encode())
    h.update(np.ascontiguousarray(nodes_r, np.float64).tobytes())
    h.update(extra.encode())
    return h.hexdigest()[:32]


def _read_record(out_dir: str) -> dict:
    path = os.path.join(out_dir, RECORD)
    if not os.path.exists(path):
        return {}
    with open(path) as fh:
        return json.load(fh)


def _write_atomic(path: str, write) -> None:
    """write(fh) into a temporary file, flushed to disk, then renamed over path."""
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        write(fh)
        fh.flush()
        os.fsync(fh.fileno())
    os.replace(tmp, path)


def batch_file(out_dir: str, b: Tuple[int, int]) -> str:
    return os.path.join(out_dir, "spectra_%05d_%05d.npz" % b)


def run(fk, params: M.FKParams, jre: int, out_dir: str, size: int = 32, resume: bool = True, log=None):
    """Compute every batch not yet recorded in ``out_dir``; returns the list of
    (batch, computed) pairs.  ``fk`` is a GeminiFK (or any object with its ``run``)."""
    os.makedirs(out_dir, exist_ok=True)
    g = M.frequency_grid(params, fk.model.rearth)
    fp = fingerprint(params, jre, fk.nodes.r)
    rec = _read_record(out_dir) if resume else {}
    if rec and rec.get("fingerprint") != fp:
        raise ValueError("%s holds batches of another run (parameters differ)" % out_dir)
    done = {tuple(b) for b in rec.get("done", [])}
    out = []
    for b in batches(g.nf1, g.nf2, size):
        if b in done and os.path.exists(batch_file(out_dir, b)):
            out.append((b, False))
            continue
        gre, gim, _, st = fk.run(params, jre, b[0], b[1], f32=True, f64=False, raise_on_failure=False)
        _write_atomic(batch_file(out_dir, b), lambda fh: np.savez(fh, gfre=gre, gfim=gim, status=st))
        done.add(b)
        rec = {"fingerprint": fp, "nf1": g.nf1, "nf2": g.nf2, "batch": size, "done": sorted(done)}
        _write_atomic(os.path.join(out_dir, RECORD), lambda fh: fh.write(json.dumps(rec).encode()))
        if log:
            log("batch %d..%d: %d items, %d failed" % (b[0], b[1], len(st), int(np.count_nonzero(st))))
        out.append((b, True))
    return out


def load(out_dir: str):
    """All recorded batches in frequency order: (gfre, gfim, status), spectra shaped
    (nnod, nsp, nkf) as GeminiFK.run returns them."""
    rec = _read_record(out_dir)
    if not rec:
        raise ValueError("%s has no completed batches" % out_dir)
    parts = [np.load(batch_file(out_dir, tuple(b))) for b in sorted(tuple(b) for b in rec["done"])]
    return (np.concatenate([p["gfre"] for p in parts], axis=2), np.concatenate([p["gfim"] for p in parts], axis=2),
            np.concatenate([p["status"] for p in parts]))


def export(out_dir: str, path: str, model, nodes, params: M.FKParams, jre: int, earth_model_name: str = "") -> None:
    """The recorded batches as one FK-spectra file (HDF5, the reference's layout),
    written batch by batch.  Every batch of the band must be recorded."""
    from .fkfile import FKFileWriter
    rec = _read_record(out_dir)
    g = M.frequency_grid(params, model.rearth)
    if not rec or rec.get("fingerprint") != fingerprint(params, jre, nodes.r):
        raise ValueError("%s holds no batches of this run" % out_dir)
    done = sorted(tuple(b) for b in rec["done"])
    covered = sum(b - a + 1 for a, b in done)
    if covered != g.nf2 - g.nf1 + 1:
        raise ValueError("only %d of the %d frequencies are recorded" % (covered, g.nf2 - g.nf1 + 1))
    with FKFileWriter(path, model, nodes, params, jre, earth_model_name=earth_model_name) as fw:
        for b in done:
            with np.load(batch_file(out_dir, b)) as z:
                fw.write_slab(b[0], b[1], z["gfre"], z["gfim"])


def main(argv=None):
    from .fk import GeminiFK
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="batched_fk", choices=sorted(configs.WORKLOADS))
    ap.add_argument("--out", required=True)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--backend", type=int, default=2, choices=[1, 2])
    ap.add_argument("--no-resume", action="store_true")
    ap.add_argument("--h5", default="", help="also write the FK-spectra file (reference HDF5 layout) to this path")
    a = ap.parse_args(argv)
    w = configs.WORKLOADS[a.workload]
    m = w.model()
    ex = w.nodes(m)
    fk = GeminiFK(m, ex, backend=a.backend)
    jre = ex.node_index(w.rec_radius)
    res = run(fk, w.params, jre, a.out, a.batch, resume=not a.no_resume, log=print)
    if a.h5:
        export(a.out, a.h5, m, ex, w.params, jre, earth_model_name=m.name)
    print(json.dumps({"batches": len(res), "computed": sum(1 for _, c in res if c)}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
