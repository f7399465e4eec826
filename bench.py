"""Benchmark of the GEMINI FK hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the batched global FK configuration -- PREM (isotropic,
no ocean), 410 frequencies to 0.2 Hz at df = 1/2048 Hz, slowness 4.0e-4 s/m,
l <= 3205, 658,944 (omega, l) solves of uneven length, 20 source radii 5..700 km
plus the surface receiver (37 external nodes after splitting).  Inputs are
synthetic model/parameter files; nothing is read from the reference.

Metric: (omega, l) ODE solves per second.  ``value`` is measured on the device
(CUDA events around the model preparation and the persistent solver, inputs
resident); ``e2e`` goes through the public C ABI with host buffers (the float32
FK spectra are copied back every step).  With N GPUs the frequencies are
split over the ranks in contiguous blocks of about equal cost, one FK launch
per rank (the reference splits them in a zig-zag order,
computeGreenFKSpectraForSynthetics.f90:361-387); the time is the maximum over
ranks.  At N > 1 the line also times the whole pipeline of one source node:
frequency-sharded FK spectra, one NCCL all-gather of that node's spectra,
station-sharded seismograms (``pipeline``).

Traces leg (``traces``): seismograms of the tensor-core degree-sum configuration
(seeded log-normal FK coefficients of the batched grid's shape, 4000 stations
x 6 moment tensors x 3 components x 8192 samples), the mixed-precision form
(sliced-integer tensor-core sums, radix-16 FFT) against the plain FP64 form,
with the relative error between the two.

``--impl reference`` times the CPU FP64 restatement of the reference (the
reference's Fortran/MPI program cannot be built here) with all host threads on
a bounded random sample of the same items.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "(ω,ℓ) ODE solves/s + seismogram traces/s on 1 B200 vs plain GPU at ≤1e-5 err"
WORKLOAD = "batched_fk"
REF_SAMPLE = 16384   # (omega, l) items of a CPU baseline step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--cpu-sample", type=int, default=0, help="items of the CPU baseline sample (0 = auto)")
    return ap.parse_args()


from gemini_unified_b200.pipeline import contiguous_runs, cost_blocks, zigzag  # noqa: E402  (frequency splits)


def sched_names(tune):
    """Autotuned schedule per phase (toroidal, spheroidal, adjoint) as
    'threads[+cache]/defer<lanes>,<steps>/q<lane run> or /qblock<block run>' strings."""
    from gemini_unified_b200.fk import DEFERRALS, GRANULARITIES, SCHEDULES
    def gran(q):
        lane, block = GRANULARITIES[q]
        return "q%d" % lane if not block else "qblock%d" % block
    return ["%d%s/defer%d,%d/%s" % (SCHEDULES[s][0], "+cache" if SCHEDULES[s][1] else "", DEFERRALS[d][0],
                                    DEFERRALS[d][1], gran(q))
            for s, d, q in zip(tune["schedule"], tune["defer"], tune["queue"])]


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_baseline(w, nsample, seed=12345, keep=False):
    """CPU FP64 oracle on a random sample of the workload's items, all host threads.
    keep: also return the sampled items and their oracle spectra [item][node][spectrum]."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from gemini_unified_b200 import model as M
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    pc = M.fk_params_c(w.params, jre)
    o = oracle.Oracle(m, ex)
    items = [(jf, iwn) for jf in range(g.nf1, g.nf2 + 1) for iwn in range(1, int(g.nwn[jf - 1]) + 1)]
    rng = np.random.default_rng(seed)
    pick = [items[i] for i in rng.choice(len(items), size=min(nsample, len(items)), replace=False)]
    ncores = os.cpu_count() or 1

    def one(it):
        jf, iwn = it
        spec = o.fk_frequency(pc, jf, int(g.nwn[jf - 1]), M.nsp_for(w.params), iwn, iwn)[0]
        return spec[:, :, iwn - 1].copy() if keep else None

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(ncores) as ex_:
        specs = list(ex_.map(one, pick))
    dt = time.perf_counter() - t
    cb = {"value": len(pick) / dt, "unit": "solves/s", "cores": ncores, "kind": "port",
          "sample": "%d (omega,l) items drawn uniformly (seed %d) from the %d of the workload; %.1f s"
                    % (len(pick), seed, len(items), dt)}
    return (cb, pick, np.stack(specs)) if keep else cb


def cpu_baseline_traces(w, g, nsp, nsta_sample, seed=12345):
    """CPU FP64 oracle of the synthetics on a random sample of the workload's stations
    (all six moment tensors, the same seeded FK coefficients and float32-rounded df and
    sigma as the GPU call), one station per host thread.  Returns the baseline, the
    sampled station indices and the oracle traces [station][mt][component][sample]."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from gemini_unified_b200 import configs
    from gemini_unified_b200.fk import synth_params
    from gemini_unified_b200.synth_run import fk_coefficients
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs)
    gr, gi = fk_coefficients(nsp, int(g.nkfmax))
    theta, phi, propdir = w.stations()
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(theta), size=min(nsta_sample, len(theta)), replace=False)
    mt = configs.unit_moment_tensors()
    ncores = os.cpu_count() or 1

    def one(i):
        return oracle.synthetics(g.nf1, g.nf2, g.nwn, g.nwnmax, sp.df, sp.sigma, gr, gi, theta[i:i + 1],
                                 phi[i:i + 1], propdir[i:i + 1], mt, w.filspecs, False, 0.0, w.nsamp, w.dt)

    t = time.perf_counter()
    with cf.ThreadPoolExecutor(ncores) as ex_:
        traces = list(ex_.map(one, pick))
    dt = time.perf_counter() - t
    ntr = len(pick) * len(mt)
    cb = {"value": ntr / dt, "unit": "traces/s", "cores": ncores, "kind": "port",
          "sample": "%d stations drawn uniformly (seed %d) from the %d of the workload, 6 moment tensors each "
                    "(%d three-component traces of %d samples); %.1f s" % (len(pick), seed, len(theta), ntr,
                                                                         w.nsamp, dt)}
    return cb, pick, np.concatenate(traces, axis=0)


def run_reference(args, rank, size):
    from gemini_unified_b200 import configs
    w = configs.WORKLOADS[args.workload]
    if rank != 0:
        return
    # the same 16,384-item sample as the cpu_baseline of the GPU arm: at 16 host
    # threads that is ~1000 items per thread, so the tail of the thread pool is
    # small against the step (a few items per thread read ~1.8x slow)
    n = args.cpu_sample or REF_SAMPLE
    for _ in range(args.warmup):
        cpu_baseline(w, max(8, n // 8), seed=1)
    vals = []
    for k in range(args.steps):
        vals.append(cpu_baseline(w, n, seed=100 + k))
    v = len(vals) * n / sum(n / x["value"] for x in vals)
    cb = dict(vals[0]); cb["value"] = v
    cb["sample"] = "%d steps of %d (omega,l) items drawn uniformly from the workload" % (len(vals), n)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": size,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n / v, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "items_per_step": n, "note": "CPU FP64 restatement of the reference"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def fk_launches_per_run(backend):
    """Kernels one gem_fk_run_device call launches: knots, splines, (Horner table,) setup, 3 phases."""
    return 6 + (1 if backend == 2 else 0)


# mixed-precision synthetics: Legendre tables, coefficients, 5 operand-slicing kernels, tensor-core sums,
# spectra, FFT twiddles, inverse FFT
SYNTH_LAUNCHES = 11


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, size)

    import ctypes
    import torch
    from gemini_unified_b200 import configs, model as M
    from gemini_unified_b200.fk import GeminiFK, synth_params, lib as fklib

    torch.cuda.set_device(local)
    dist = None
    if size > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def max_over_ranks(v):
        if not dist:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = configs.WORKLOADS[args.workload]
    m = w.model()
    ex = w.nodes(m)
    jre = ex.node_index(w.rec_radius)
    g = M.frequency_grid(w.params, m.rearth)
    nsp = M.nsp_for(w.params)
    # one contiguous block of frequencies of about equal cost per rank: one FK launch
    # each (the reference's zig-zag order gives a rank many short runs)
    runs = cost_blocks(g.nwn, g.nf1, g.nf2, size)[rank]
    dev = torch.device("cuda", local)
    nkf = {r: int(g.nwn[r[0] - 1: r[1]].sum()) for r in runs}
    items_rank = sum(nkf.values())
    biggest = max(nkf.values())
    n_out = biggest * nsp * ex.nnod
    gre = torch.empty(n_out, dtype=torch.float32, device=dev)
    gim = torch.empty(n_out, dtype=torch.float32, device=dev)
    gst = torch.empty(biggest, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    total_items = int(g.nkfmax)

    phase = {"flops": [0, 0, 0], "ms": [0.0, 0.0, 0.0]}

    def fk_step(fk, keep=None):
        flops = 0
        phase["flops"], phase["ms"] = [0, 0, 0], [0.0, 0.0, 0.0]
        for r in runs:
            fk.run_device(w.params, jre, r[0], r[1], gfre=gre.data_ptr(), gfim=gim.data_ptr(),
                          status=gst.data_ptr(), stream=stream.cuda_stream)
            s = fk.stats()
            flops += s["flops"]
            for i in range(3):
                phase["flops"][i] += s["phase_flops"][i]
                phase["ms"][i] += s["phase_ms"][i]
            if int(gst[: nkf[r]].abs().sum()) != 0:
                raise RuntimeError("failed (omega,l) items in frequencies %d..%d" % r)
            if keep is not None:
                keep(r)
        return flops

    def timed(fn, steps, clocks=None):
        times, out = [], None
        for _ in range(steps):
            flush.fill_(1.0)
            if dist: dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = fn()
            e1.record(stream)
            torch.cuda.synchronize()
            if dist: dist.barrier()
            times.append(e0.elapsed_time(e1))
        return max_over_ranks(float(np.mean(times))), out

    # ---------------- batched + mixed-precision form (fast FP64 build): the headline
    fast = GeminiFK(m, ex, device=local, backend=2)
    # the autotuner picks each phase's schedule (block size, matrix caching) and
    # bookkeeping deferral on the whole band, untimed.  On the top quarter alone the two
    # best spheroidal schedules differ by less than the run-to-run noise (262 against
    # 265 ms) while over the whole band they differ by 5% (380 against 399 ms).
    tune_fast = fast.autotune(w.params, jre, g.nf1, g.nf2)
    for _ in range(args.warmup):
        fk_step(fast)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    t_ms, flops_step = timed(lambda: fk_step(fast), args.steps)
    clk = clocks.stop()
    sph_flops, sph_ms = phase["flops"][1], max_over_ranks(phase["ms"][1])
    phase_ms_fast = list(phase["ms"])
    value = total_items / (t_ms / 1e3)

    # ---------------- plain FP64 form (reference rounding, one operation at a time)
    plain = GeminiFK(m, ex, device=local, backend=1)
    tune_plain = plain.autotune(w.params, jre, g.nf1, g.nf2)
    fk_step(plain)
    plain_steps = max(1, min(args.steps, 2))
    t_plain, _ = timed(lambda: fk_step(plain), plain_steps)
    plain_value = total_items / (t_plain / 1e3)
    del plain

    # ---------------- end-to-end through the host C ABI (float32 spectra back to pinned host buffers)
    host_out = {r: tuple(torch.empty((ex.nnod, nsp, nkf[r]), dtype=torch.float32, pin_memory=True).numpy()
                         for _ in range(2)) for r in runs}
    for r in runs:   # warm-up: the context's device buffers of the host entry point
        fast.run(w.params, jre, r[0], r[1], f32=True, f64=False, out=host_out[r])
    e2e_times = []
    for _ in range(max(1, min(args.steps, 2))):
        if dist: dist.barrier()
        t0 = time.perf_counter()
        for r in runs:
            fast.run(w.params, jre, r[0], r[1], f32=True, f64=False, out=host_out[r])
        e2e_times.append(time.perf_counter() - t0)
    del host_out
    e2e_s = max_over_ranks(float(np.mean(e2e_times)))
    d2h = items_rank * nsp * ex.nnod * 4 * 2 + items_rank * 4
    h2d = items_rank * 8 + 9 * (m.nk + 1) * 8

    # ---------------- seismogram traces: FK spectra of one source node -> traces at all stations
    traces = time_traces(args, w, m, g, nsp, dev, stream, dist, rank, size, timed)
    # ---------------- N GPUs: frequency-sharded FK -> one all-gather -> station-sharded traces
    pipe = time_pipeline(w, m, ex, jre, g, nsp, local, dev, stream, rank, size, timed) if size > 1 else None

    # ---------------- roofline of the dominant kernel: the spheroidal phase (FP64 pipe)
    peak = fp64_peak_tflops(local)
    achieved = sph_flops / (sph_ms / 1e3) / 1e12
    traffic = None
    prof = os.path.join(ROOT, "profiles", "fk_phase_sph_batched_fk.json")
    if os.path.exists(prof):
        pj = json.load(open(prof))
        traffic = pj["dram_bytes_per_item"] * items_rank

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (PREM node model from the reference's data files; seeded inputs)",
            "config": {"workload": args.workload, "solves_per_step": total_items, "frequencies": int(g.nf2 - g.nf1 + 1),
                       "lmax": int(g.nwn.max() - 1), "nodes": int(ex.nnod), "parallelism": "frequency zig-zag over %d GPU(s)" % size,
                       "form": "fast FP64 build (FMA, Horner spline table, reciprocals); batched phase kernels",
                       "schedule": {"fast": sched_names(tune_fast), "plain": sched_names(tune_plain),
                                    "tuned_on_jf": tune_fast["jf"]},
                       "l2": "flushed between steps (256 MiB write); outputs (1.9 GB) exceed L2"},
            "plain_fp64": {"value": plain_value, "unit": "solves/s", "ms_per_step": t_plain, "steps": plain_steps,
                           "speedup_of_value": value / plain_value},
            "traces": traces,
            "roofline": {"kernel": "gem_fast::fk_phase_kernel<1> (spheroidal minors)", "bound": "fp64",
                         "achieved": achieved, "peak": peak["tflops"], "unit": "TFLOP/s",
                         "frac": achieved / peak["tflops"], "traffic": traffic, "peak_source": peak["source"],
                         "flops_per_launch": sph_flops, "launch_ms": sph_ms, "phase_ms": phase_ms_fast,
                         "step_flops": flops_step, "step_tflops": flops_step / (t_ms / 1e3) / 1e12,
                         "flops_note": "reference-algorithm FP64 flops (cached system matrices, full Neville) counted per event on the device; traffic scaled from an ncu capture of the 8 highest frequencies"},
            "e2e": {"value": total_items / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": fk_launches_per_run(2) * len(runs) * args.steps,
            "gpu_launches_traces": SYNTH_LAUNCHES * traces.pop("steps_timed", max(1, min(args.steps, 3))),
            "clocks": clk,
        }
        if pipe is not None:
            line["pipeline"] = pipe
        out_fast = line["traces"].pop("_out")
        if size == 1:
            n = args.cpu_sample or REF_SAMPLE
            cb, pick, ref = cpu_baseline(w, n, keep=True)
            line["cpu_baseline"] = cb
            fk_step(fast)   # untimed: the plain form's timing overwrote the output buffers
            torch.cuda.synchronize()
            line["error_vs_oracle"] = fk_error_vs_oracle(g, nsp, ex.nnod, gre, gim, pick, ref)
            cbt, sta, ref_tr = cpu_baseline_traces(w, g, nsp, 1024)
            line["traces"]["cpu_baseline"] = cbt
            from gemini_unified_b200.synth_run import trace_errors
            line["traces"]["error_vs_oracle"] = dict(
                trace_errors(out_fast[torch.as_tensor(sta, device=dev)], torch.from_numpy(ref_tr).to(dev)),
                stations=len(sta), note="mixed form of the timed run against the CPU FP64 oracle on the sampled "
                                        "stations (all six moment tensors)")
        del out_fast
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def time_pipeline(w, m, ex, jre, g, nsp, local, dev, stream, rank, size, timed):
    """The FK-to-seismogram pipeline of the 5 km source node on N GPUs
    (gemini_unified_b200.pipeline): each rank computes the FK spectra of its
    block of frequencies (all nodes, fast form), one NCCL all-gather brings the
    source node's float32 spectra of every frequency to every rank, and each
    rank computes the seismograms of its share of the 4000 stations (mixed
    form).  Timed as one step, the maximum over ranks."""
    from gemini_unified_b200 import configs, pipeline as P
    from gemini_unified_b200.fk import synth_params
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs)
    mt = configs.unit_moment_tensors()
    st = P.GpuStages(m, ex, w.params, jre, sp, w.stations(), mt, device=local, backend=2, stream=stream)
    src = ex.node_index(m.rearth - 5000.0)
    nsta = w.ndist

    def one():
        return P.fk_to_traces(rank, size, g.nwn, g.nf1, g.nf2, nsp, src, nsta, st.fk_fn, st.synth_fn, device=dev)

    one()   # warm-up: buffers of the context
    t_ms, _ = timed(one, 1)
    return {"ms_per_step": t_ms, "unit": "ms", "source_node": int(src), "stations": nsta, "moment_tensors": len(mt),
            "partition": "cost-balanced frequency blocks, stations round robin",
            "allgather_bytes_per_rank": int(2 * nsp * P.SlabPartition(g.nwn, g.nf1, g.nf2, P.cost_blocks(
                g.nwn, g.nf1, g.nf2, size)).width * 4),
            "slab_bytes": int(2 * nsp * int(g.nkfmax) * 4)}


def fk_error_vs_oracle(g, nsp, nnod, gre, gim, pick, ref):
    """float32 spectra of the timed run (device, Fortran order (nkf, nsp, nnod)) against the
    CPU FP64 oracle on the sampled items: |gpu - oracle| relative to the largest value of each
    spectrum (node, component) of the item's frequency, over all the sample's values."""
    import torch
    nkf = int(g.nkfmax)
    gr = gre[: nkf * nsp * nnod].view(nnod, nsp, nkf)
    gi = gim[: nkf * nsp * nnod].view(nnod, nsp, nkf)
    koff = np.concatenate([[0], np.cumsum(g.nwn[g.nf1 - 1: g.nf2])]).astype(np.int64)
    jfs = sorted({jf for jf, _ in pick})
    scale = {}
    for jf in jfs:
        a, b = int(koff[jf - g.nf1]), int(koff[jf - g.nf1 + 1])
        mag = torch.sqrt(gr[:, :, a:b].double() ** 2 + gi[:, :, a:b].double() ** 2)
        scale[jf] = torch.nan_to_num(mag, nan=0.0).amax(dim=-1).cpu().numpy()
    ks = np.array([koff[jf - g.nf1] + iwn - 1 for jf, iwn in pick], np.int64)
    kt = torch.as_tensor(ks, device=gre.device)
    got = (gr[:, :, kt].double().cpu().numpy() + 1j * gi[:, :, kt].double().cpu().numpy()).transpose(2, 0, 1)
    sc = np.stack([scale[jf] for jf, _ in pick])
    nan_ok = bool(np.array_equal(np.isnan(got), np.isnan(ref)))
    ok = ~np.isnan(ref) & (sc > 0)
    rel = np.abs(got - ref)[ok] / sc[ok]
    return {"items": len(pick), "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
            "nan_positions_equal": nan_ok,
            "note": "float32 spectra of the timed fast run against the CPU FP64 oracle (float32 rounding is "
                    "6e-8); the FP64 outputs are held to 1e-8 by the GPU tests"}


def time_traces(args, w, m, g, nsp, dev, stream, dist, rank, size, timed):
    """Seismogram traces of the tensor-core degree-sum configuration: seeded
    log-normal FK coefficients of the batched grid's shape (nsp x 658,944,
    l <= 3205), 4000 stations 0.5..179.5 deg x 6 unit moment tensors, 3
    components of 8192 samples.  The mixed-precision form (sliced-integer
    tensor-core sums, radix-16 inverse FFT) against the plain FP64 form.  With
    N ranks the stations are split over the ranks."""
    import ctypes
    import torch
    from gemini_unified_b200 import configs
    from gemini_unified_b200.fk import FrequencyTime, lib as fklib, synth_params
    from gemini_unified_b200.synth_run import fk_coefficients, trace_errors
    gr_h, gi_h = fk_coefficients(nsp, int(g.nkfmax))
    d_gr = torch.from_numpy(gr_h).to(dev)
    d_gi = torch.from_numpy(gi_h).to(dev)
    theta, phi, propdir = w.stations()
    sel = slice(rank, None, size)
    theta, phi, propdir = [np.ascontiguousarray(a[sel]) for a in (theta, phi, propdir)]
    mt = np.ascontiguousarray(configs.unit_moment_tensors(), np.float64)
    nsta, nmt = len(theta), len(mt)
    sp = synth_params(g, nsp, w.nsamp, w.dt, w.filspecs)
    nwn = np.ascontiguousarray(g.nwn, np.int32)
    L = fklib()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    ntr = w.ndist * nmt

    def form(backend, steps):
        ctx = FrequencyTime(device=dev.index, backend=backend)
        out = torch.empty((nsta, nmt, 3, w.nsamp), dtype=torch.float32, device=dev)

        def one():
            rc = L.gem_synth_run_device(ctx._h, ctypes.byref(sp), p(nwn), d_gr.data_ptr(), d_gi.data_ptr(), nsta,
                                        p(theta), p(phi), p(propdir), nmt, p(mt), out.data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream))
            if rc >= 2:
                raise RuntimeError(L.gem_last_error(ctx._h).decode())

        for _ in range(max(1, args.warmup - 1)):
            one()
        t_ms, _ = timed(one, steps)
        return ctx, out, t_ms

    fast_ctx, out_fast, t_fast = form(2, max(1, min(args.steps, 3)))
    _, out_plain, t_plain = form(1, 1)
    err = trace_errors(out_fast, out_plain)
    # end to end through the host C ABI: FK coefficients from pinned host memory, traces back to it
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    gr_p, gi_p = pin(gr_h), pin(gi_h)
    tr_h = torch.empty((nsta, nmt, 3, w.nsamp), dtype=torch.float32, pin_memory=True).numpy()

    def host_call():
        rc = L.gem_synth_run(fast_ctx._h, ctypes.byref(sp), p(nwn), p(gr_p), p(gi_p), nsta, p(theta), p(phi),
                             p(propdir), nmt, p(mt), p(tr_h))
        if rc >= 2:
            raise RuntimeError(L.gem_last_error(fast_ctx._h).decode())

    host_call()   # warm-up: the context's device buffers of the host entry point
    e2e_runs = []
    for _ in range(max(1, min(args.steps, 3))):
        if dist: dist.barrier()
        t0 = time.perf_counter()
        host_call()
        e2e_runs.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_runs))
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    return {"value": ntr / (t_fast / 1e3), "unit": "traces/s", "ms_per_step": t_fast, "traces_per_step": ntr,
            "samples": w.nsamp, "components": 3, "stations": w.ndist, "moment_tensors": nmt,
            "data": "seeded log-normal FK coefficients, log10|c| ~ N(-3, 1) clipped to [-6, 0], uniform phase",
            "form": "sliced-INT8 degree sums on tcgen05 (exact INT32 accumulation) + real-output radix-16 FP64 inverse FFT",
            "plain_fp64": {"value": ntr / (t_plain / 1e3), "unit": "traces/s", "ms_per_step": t_plain,
                           "form": "FP64 tiled degree-sum products (CUDA cores) + reference radix-2 inverse FFT",
                           "speedup_of_value": t_plain / t_fast},
            "error_vs_plain_fp64": err,
            "_out": out_fast,
            "e2e": {"value": ntr / e2e_s, "unit": "traces/s", "h2d_bytes_per_step": int(gr_h.nbytes * 2),
                    "d2h_bytes_per_step": int(tr_h.nbytes)}}


def fp64_peak_tflops(device):
    """FP64 FMA throughput measured with the benchmark's own probe kernel (this run);
    the probe lives in libgem_bench_probe.so, outside the product library."""
    import ctypes
    from gemini_unified_b200 import build
    try:
        f = ctypes.CDLL(build.PROBE_LIB).gem_probe_fp64_tflops
    except (OSError, AttributeError):
        return {"tflops": 37.0, "source": "nominal B200 FP64 (no probe)"}
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_int]
    v = f(device)
    if not v > 0:
        return {"tflops": 37.0, "source": "nominal B200 FP64 (probe failed)"}
    return {"tflops": v, "source": "measured in this run: FP64 FMA-chain probe kernel, all SMs"}


if __name__ == "__main__":
    main()
