"""Throughput benchmark: chi2 evaluations per second (target x z x template).

Workload (one "step", default ``uneven5000``): 5000 synthetic DESI-like
targets (cameras b/r/z, P = 7958 pixels, 11-diagonal resolution with its
width varying per camera, 0-40 % of pixels masked per target, 10 % of the
targets with one camera dropped) scanned against the full template set --
GALAXY (10 bases, 3311 z), QSO (4 bases, 3794 z, Inoue14 IGM) and 5 STAR
subtypes (5 bases, 100 z) -- i.e. 7605 chi2 evaluations per target, 38.0 M
per step.  A step runs the whole hot path: rebin + IGM bases for every
template, target packing, the tensor-core y GEMM and the fused scan (chi2,
coefficients and [OII] penalty for every target, template and z).  The
500-target batch (``desi500``, 5 % masked) is reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): every rank scans its own targets
(weak scaling, no collective in the data path); the step time is the max
over ranks.  ``--impl reference`` times redrock's own CPU path (the
unmodified install at baseline/_ref: DistTemplate construction, then
calc_zchi2_targets with one process per host core) on a sample of the same
workload, or the CPU restatement in oracle/ when that install is absent.
"""

from __future__ import annotations

import argparse
import contextlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

D_BAND = 11
WORKLOAD_NAMES = {
    "desi500": "zscan-desi-500x(GALAXY3311+QSO3794+5xSTAR100)",
    "uneven5000": "zscan-uneven-5000x(GALAXY3311+QSO3794+5xSTAR100): 0-40% masked, "
                  "10% one camera dropped, resolution width per camera",
    "stress20000": "zscan-stress-20000x(GALAXY3311+QSO3794+5xSTAR100): 60% QSO-like z<=6 "
                   "with Inoue14, S/N 0.5-50",
}
DEFAULT_WORKLOAD = "uneven5000"
METRIC = "chi2 evals/s (target x z x template) on 1 B200, fused vs plain, |dchi2|<=1e-3"


def flops_per_eval(nb, npix):
    """Algorithmic FLOPs of one chi2 evaluation in redrock's formulation:
    R.T (2 D P n), weighted Gram (P n (n+1)), y (2 P n), solve (n^3/3 + 2n^2),
    chi2 via b.c (2n)."""
    return npix * nb * (2 * D_BAND + nb + 3) + nb ** 3 / 3.0 + 2 * nb ** 2 + 2 * nb


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
WORKLOADS = {
    # the 500-target DESI-like batch (the headline)
    "desi500": dict(ntarget=500),
    # uneven batching: 0-40 % of pixels masked per target, 10 % of targets
    # with one camera dropped, resolution width varying per camera
    "uneven5000": dict(ntarget=5000, mask_range=(0.0, 0.4), drop_camera_frac=0.1),
    # precision stress: 60 % QSO-like targets at z up to 6 rendered with
    # Inoue14 IGM attenuation, S/N (amplitude) log-uniform 0.5-50
    "stress20000": dict(ntarget=20000, qso_frac=0.6, snr_range=(0.5, 50.0)),
}


def synth_targets(workload, n, seed, transmission=None):
    """Seeded synthetic targets of a workload (plain numpy)."""
    from redrock_b200 import synth
    spec = dict(WORKLOADS[workload])
    spec.pop("ntarget", None)
    if "qso_frac" in spec:
        return synth.make_population(n, seed=seed, transmission=transmission, **spec)
    return synth.make_targets(n, seed=seed, **spec)


def make_workload(ntarget, seed, zsub=None, workload=DEFAULT_WORKLOAD):
    from redrock_b200 import synth
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    n = ntarget or WORKLOADS[workload]["ntarget"]
    tr = None
    if "qso_frac" in WORKLOADS[workload]:
        from redrock_b200.igm import transmission_Lyman

        def tr(z, w):
            return transmission_Lyman(np.array([z]), w, model="Inoue14")[0]
    tg = synth_targets(workload, n, seed, transmission=tr)
    tset = synth.template_set(zsub=zsub)
    rtg = T.from_synth(tg)
    tms = [TM.from_synth(ts) for ts in tset]
    return tg, rtg, tset, tms


def evals_and_flops(rtg, tms):
    """(evals, algorithmic FLOPs F(n, P) summed, the y part 2 P n of them)"""
    ev = 0
    fl = 0.0
    yfl = 0.0
    for t in rtg:
        npix = sum(len(s.wave) for s in t.spectra)
        for tm in tms:
            nz = len(tm.redshifts)
            ev += nz
            fl += nz * flops_per_eval(tm.nbasis, npix)
            yfl += nz * 2.0 * npix * tm.nbasis
    return ev, fl, yfl


def measure_fp64_peak(L, torch):
    from redrock_b200.device import stream_handle
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = nsm * 8, 2000
    L.rr_fma_peak(0, blocks, iters, out.data_ptr(), stream_handle())
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        L.rr_fma_peak(0, blocks, iters, out.data_ptr(), stream_handle())
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        best = max(best, 2.0 * 8 * 16 * iters * blocks * 256 / t / 1e12)
    return best


def traffic_from_profile(workload, reduced):
    """DRAM bytes per launch of the fused scan kernel from the committed ncu
    summary (profiles/zscan_fused_traffic.json), for the workload it was
    captured on (desi500 at full size) only."""
    p = os.path.join(ROOT, "profiles", "zscan_fused_traffic.json")
    if workload == "desi500" and not reduced and os.path.exists(p):
        try:
            return json.load(open(p)).get("bytes_per_launch_full_workload")
        except Exception:
            return None
    return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from redrock_b200 import _lib, synth, zscan
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    from redrock_b200.device import StatusWord
    from redrock_b200.engine import (DeviceBasis, GridLayout, TargetBatch, TargetPack,
                                     TemplateSource, run_fused)

    torch.cuda.set_device(local_rank)
    L = _lib.lib()
    tg, rtg, tset, tms = make_workload(args.ntargets, seed=args.seed + 7919 * rank,
                                       zsub=args.zsub, workload=args.workload)
    evals, flops, y_flops = evals_and_flops(rtg, tms)
    layout = GridLayout.from_dwave(synth.camera_grids())
    if args.ygemm is None:
        # the engine's own choice for this layout (what the public API runs)
        from redrock_b200.engine import resolve_y
        args.ygemm = resolve_y(None, layout)
    srcs = [TemplateSource.from_template(tm) for tm in tms]
    dbatch = TargetBatch(rtg, layout).to_device()
    bases_gb = sum(len(tm.redshifts) * layout.pix_stride * (tm.nbasis + tm.nbasis % 2) * 8
                   for tm in tms) / 1e9
    pack_gb = dbatch.batch.nblock * dbatch.batch.npix_block * _lib.RW * _lib.LANES * 8 / 1e9
    st = StatusWord()
    ev_fused = []

    ev_kernel = []

    tiles = None
    tuned = None
    if args.tiles:
        # a fixed tile choice (e.g. the one an earlier run's autotuner made)
        tiles = {(int(k) if k.isdigit() else k): int(v) for k, v in json.loads(args.tiles).items()}
    elif args.autotune:
        # tile shapes picked by the autotuner before anything is timed
        from redrock_b200 import autotune
        bases0 = [DeviceBasis.build(s, layout, status=st) for s in srcs]
        pack0 = TargetPack(dbatch, status=st)
        tuned = autotune.tune(pack0, bases0)
        tiles = autotune.tiles_of(tuned)
        del bases0, pack0

    def step(record, ygemm=args.ygemm, sink=ev_fused, external=False):
        bases = [DeviceBasis.build(s, layout, status=st) for s in srcs]
        pack = TargetPack(dbatch, status=st)
        if record:
            e0 = torch.cuda.Event(enable_timing=True, external=external)
            e1 = torch.cuda.Event(enable_timing=True, external=external)
            e0.record()
        res, _ = run_fused(pack, bases, status=st, ygemm=ygemm,
                           kernel_events=ev_kernel if (record and sink is ev_fused) else None,
                           tiles=tiles, external_events=external)
        if record:
            e1.record()
            sink.append((e0, e1))
        return res, pack

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    st.check("warm-up")
    graph = None
    if args.graph:
        # the whole step (basis launches, packing, y GEMM, the fused scan) as
        # one CUDA graph, replayed per step; its timing events are graph
        # nodes, so every replay re-times the scan stage and the fused
        # launches (the values read after the timed region are the last
        # replay's)
        from redrock_b200.device import capture_graph
        graph, _ = capture_graph(lambda: step(True, external=True))
        graph.replay()
        torch.cuda.synchronize()
        st.check("graph replay")
    # basis builds, target packing (2), one fused launch per nbasis group;
    # with a tensor-core y also the G packing, slicing and one GEMM per
    # template
    groups = {0 if tm.nbasis == 10 else 1 if tm.nbasis == 4 else 2 if tm.nbasis == 5 else 3
              for tm in tms}
    launches_per_step = sum(len(layout.keys) for _ in srcs) + 2 + len(groups)
    if args.ygemm in ("int8x7", "int8x6"):
        # rr_pack_g, rr_slice_g_i8; per template rr_basis_col_exp,
        # rr_slice_basis_i8, rr_ygemm_i8
        launches_per_step += 2 + 3 * len(srcs)
    elif args.ygemm != "fp64":
        launches_per_step += 1 + len(srcs)

    clocks = ClockSampler(torch.cuda.current_device())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        if graph is not None:
            graph.replay()
        else:
            step(True)
    t1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    st.check("timed steps")
    ms = t0.elapsed_time(t1) / args.steps
    resweeps = resweep_lanes = None
    if hasattr(run_fused, "last_counter"):
        resweeps = int(run_fused.last_counter[2].item())
        resweep_lanes = int(run_fused.last_counter[3].item())
    # scan stage (y GEMM + fused kernel) and the fused kernel alone
    timing_note = ("CUDA events in the captured graph: scan stage and fused launches of the "
                   "last timed replay" if graph is not None else
                   "CUDA events around the scan stage and the fused launches of every timed step")
    try:
        fused_ms = float(np.mean([a.elapsed_time(b) for a, b in ev_fused])) if ev_fused else ms
        kernel_ms = (float(np.mean([a.elapsed_time(b) for a, b in ev_kernel])) * len(ev_kernel)
                     / max(len(ev_fused), 1)) if ev_kernel else fused_ms
    except RuntimeError:
        # events recorded by graph nodes not readable here: time one eager
        # step right after the timed region instead
        ev_fused.clear()
        ev_kernel.clear()
        step(True)
        torch.cuda.synchronize()
        fused_ms = float(np.mean([a.elapsed_time(b) for a, b in ev_fused]))
        kernel_ms = float(np.sum([a.elapsed_time(b) for a, b in ev_kernel]))
        timing_note = "CUDA events around one eager step right after the timed graph replays"
    if world > 1:
        v = torch.tensor([ms, fused_ms, kernel_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
        ms, fused_ms, kernel_ms = float(v[0]), float(v[1]), float(v[2])
    value = world * evals / (ms / 1e3)

    study = ygemm_study(args, step, torch, evals) if args.ygemm_study else None
    adj = adjoint_study(rtg, tms, torch) if (args.adjoint and rank == 0) else None
    zst = zfind_study(rtg, tms, torch, ntarget=args.zfind_targets) \
        if (args.zfind and rank == 0) else None
    arc = archetype_study(tg, rtg, torch) if (args.archetypes and rank == 0) else None

    # ---- end to end through the public API, host buffers ------------------
    e2e = None
    if not args.no_e2e:
        def e2e_step():
            zscan.clear_caches()
            dtg = T.DistTargetsCopy(rtg)
            dwave = dtg.wavegrids()
            dts = [TM.DistTemplate(tm, dwave) for tm in tms]
            res = zscan.calc_zchi2_targets(dtg, dts)
            return res
        # calc_zchi2_targets prints redrock's progress line; keep stdout for
        # the one JSON result line
        with contextlib.redirect_stdout(sys.stderr):
            for _ in range(max(1, min(args.warmup, 2))):
                e2e_step()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            n_e2e = max(1, min(args.steps, args.e2e_steps))
            a.record()
            for _ in range(n_e2e):
                e2e_step()
            b.record()
        torch.cuda.synchronize()
        e2e_ms = a.elapsed_time(b) / n_e2e
        if world > 1:
            v = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(v, op=dist.ReduceOp.MAX)
            e2e_ms = float(v[0])
        batch = TargetBatch(rtg, layout)
        h2d = batch.nbytes + sum(s.nbytes for s in srcs) + sum(
            2 * 8 * (n + 1) for n in layout.npix)
        d2h = sum(len(rtg) * len(tm.redshifts) * (2 + tm.nbasis) * 8 for tm in tms)
        e2e = {"value": world * evals / (e2e_ms / 1e3), "unit": "chi2 evals/s",
               "ms_per_step": e2e_ms, "steps": n_e2e, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": "redrock_b200.zscan.calc_zchi2_targets(DistTargetsCopy, [DistTemplate x7])"
                       " from host numpy arrays"}

    # ---- plain per-target chain on a sample (the "plain" of fused vs plain)
    plain = None
    if not args.no_plain and rank == 0:
        sample = rtg[:args.plain_targets]
        dtg = T.DistTargetsCopy(sample)
        dts = [TM.DistTemplate(tm, dtg.wavegrids()) for tm in tms]
        ids = [t.id for t in sample]
        zscan.calc_zchi2_plain(ids[:1], sample[:1], dts[0])    # warm-up
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for dt in dts:
            zscan.calc_zchi2_plain(ids, sample, dt)
        b.record()
        torch.cuda.synchronize()
        pev = len(sample) * sum(len(tm.redshifts) for tm in tms)
        pv = pev / (a.elapsed_time(b) / 1e3)
        plain = {"value": pv, "unit": "chi2 evals/s", "targets": len(sample),
                 "fused_over_plain": (evals / (ms / 1e3)) / pv,
                 "path": "redrock_b200.zscan.calc_zchi2_plain: per target and template, "
                         "R.T -> Gram/y -> solve -> residual chi2 launches + host read-back"}

    if rank != 0:
        return None
    peak = measure_fp64_peak(L, torch)
    # FP64 work of the fused kernel: all of F(n, P), less y when the tensor
    # cores compute it
    y_on_tc = args.ygemm != "fp64"
    fused_flops = flops - (y_flops if y_on_tc else 0.0)
    achieved = fused_flops / (kernel_ms / 1e3) / 1e12
    out = {
        "metric": METRIC,
        "value": value, "unit": "chi2 evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded DESI-like targets and "
        "templates, redrock_b200/synth.py)",
        "config": {"workload": WORKLOAD_NAMES[args.workload]
                   if not args.ntargets and not args.zsub else
                   f"reduced {args.workload}: {len(rtg)} targets, zsub={args.zsub}",
                   "targets_per_gpu": len(rtg),
                   "templates": [tm.full_type for tm in tms],
                   "evals_per_step_per_gpu": evals,
                   "pixels_per_target": "7958 (fewer with a dropped camera)",
                   "l2": (f"inputs larger than L2 (bases {bases_gb:.1f} GB + packed targets "
                          f"{pack_gb:.2f} GB per step; L2 126 MB)"),
                   "parallelism": f"targets sharded {world}-way, no collective",
                   "cuda_graph": bool(args.graph),
                   "y_term": args.ygemm,
                   "tile": {"targets": 32, "redshifts_per_thread": tiles or "default (nbasis 4, 5: 2)",
                            "warps": 8, "pixels_per_stage": 24,
                            "chosen_by": ("autotuner (kernel time per candidate, ms: "
                                          + str({k: v for k, v in tuned.items()
                                                 if not isinstance(k, int)}) + ")")
                            if tuned else ("--tiles" if args.tiles else "defaults")}},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic_from_profile(args.workload,
                                                                  bool(args.ntargets or args.zsub)),
                     "traffic_note": (
                         "desi500: DRAM bytes of the three group launches from a full-size "
                         "ncu capture (profiles/zscan_fused_traffic.json)"
                         if args.workload == "desi500" else
                         "not scaled from a small case: the L2 reuse of packed rows depends on "
                         "how many running tiles share a target block; small-case bytes per tile "
                         "and the bounds for the full launch in "
                         "profiles/zscan_fused_traffic_uneven640.md"),
                     "kernel": "zscan_fused_kernel",
                     "kernel_ms": kernel_ms, "flops_per_launch": fused_flops,
                     "flops_note": ("FP64 FLOPs of F(n,P) done by this kernel"
                                    + ("; y (2 P n per eval) on the tensor cores" if y_on_tc
                                       else "")),
                     "scan_stage_ms": fused_ms,
                     "kernel_timing": timing_note,
                     "resweep_tiles_per_launch": resweeps,
                     "resweep_evals_per_launch": resweep_lanes,
                     "peak_source": "measured FP64 FMA peak (rr_fma_peak) on this GPU"},
        "e2e": e2e,
        "plain": plain,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if study is not None:
        out["ygemm_study"] = study
    if adj is not None:
        out["adjoint"] = adj
    if zst is not None:
        out["zfind"] = zst
    if arc is not None:
        out["archetypes"] = arc
    return out


def zfind_study(rtg, tms, torch, ntarget=500):
    """zfind on the first ntarget targets of the workload against all 7
    templates (3 minima each; config 2's 500 x 7 x 3 by default): wall time
    of the eager path, of the CUDA-graph path (scan, then each template's
    candidates + fine grids, as captured graphs) and of batched Newton
    refinement; and, for every target's best
    GALAXY minimum with ZWARN 0, the distance of the parabola and Newton
    redshifts to the minimum of a dense FP64 scan (401 points spanning two
    fine-grid steps around it, rr_zscan_pairs)."""
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.engine import RowPack, TemplateSource, run_pairs
    from redrock_b200.zfind import zfind
    sub = rtg[:ntarget]
    dz = T.DistTargetsCopy(sub)
    dts = [TM.DistTemplate(tm, dz.wavegrids()) for tm in tms]

    def timed(**kw):
        # the first call includes the one-time set-up (autotuner, device
        # packs; with graph=True the plan's buffers and the capture), the
        # second reuses what is cached for the same objects
        from redrock_b200.zscan import clear_caches
        with contextlib.redirect_stdout(sys.stderr):
            clear_caches()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            zfind(dz, dts, nminima=3, **kw)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            out = zfind(dz, dts, nminima=3, **kw)
            torch.cuda.synchronize()
        return time.perf_counter() - t1, out[1], t1 - t0
    t_eager, par, t_eager1 = timed()
    t_graph, gra, t_graph1 = timed(graph=True)
    t_newton, new, t_newton1 = timed(refine="newton")
    same = all(np.array_equal(np.asarray(gra[k]), np.asarray(par[k])) for k in par)
    # dense FP64 scans of the fine-grid cell each target's best GALAXY
    # minimum was refined in (the three fine-grid points around the best)
    gal = tms[0]
    src = TemplateSource.from_template(gal)
    rows = RowPack.from_targets(sub, dts[0].basis.layout)
    zgrid = np.asarray(gal.redshifts)
    fine = 2.0 * np.median(np.diff(np.log1p(zgrid))) / 14
    err_p, err_n = [], []
    idx = {t.id: i for i, t in enumerate(sub)}
    for tab, errs in ((par, err_p), (new, err_n)):
        m = np.nonzero((tab["znum"] == 0) & (tab["spectype"] == "GALAXY")
                       & (tab["zwarn"] == 0))[0]
        if len(m) == 0:
            continue
        zs = tab["z"][m]
        k = np.clip(np.argmin(tab["zzchi2"][m], axis=1), 1, tab["zz"].shape[1] - 2)
        zd = np.linspace(tab["zz"][m, k - 1], tab["zz"][m, k + 1], 401, axis=1)
        pt = np.repeat([idx[t] for t in tab["targetid"][m]], 401).astype(np.int32)
        c2, _, pen = run_pairs(rows, src, pt, zd.ravel())
        c2 = (c2 + pen).cpu().numpy().reshape(len(m), 401)
        zbest = zd[np.arange(len(m)), np.argmin(c2, axis=1)]
        # chi2 of the reported minimum: the parabola's is its fitted vertex,
        # so it is evaluated at the reported z here for both
        zrep = np.asarray(zs, dtype=np.float64)
        cr, _, penr = run_pairs(rows, src, np.array([idx[t] for t in tab["targetid"][m]],
                                                    dtype=np.int32), zrep)
        cr = (cr + penr).cpu().numpy()
        # (|dln(1+z)| to the dense minimum, chi2 at the reported z minus the
        # dense minimum's chi2)
        errs.extend(zip(np.abs(np.log1p(zs) - np.log1p(zbest)).tolist(),
                        (cr - c2.min(axis=1)).tolist()))
    return {"targets": len(sub), "templates": len(tms), "nminima": 3,
            "eager_s": t_eager, "graph_s": t_graph, "newton_s": t_newton,
            "first_call_s": {"eager": t_eager1, "graph": t_graph1, "newton": t_newton1},
            "timing": "second call on the same objects (device packs, and with graph=True the "
                      "captured plan, reused: the graph is replayed); first_call_s includes the "
                      "set-up",
            "graph_equals_eager": bool(same),
            "dense_grid_check": dict(
                cases=len(err_n), grid="401 points over the refined fine-grid cell (FP64)",
                dense_grid_step_dlnz=float(2 * fine / 400),
                **{f"{k}_{name}": (float(f(np.asarray(e)[:, col])) if e else None)
                   for name, e in (("parabola", err_p), ("newton", err_n))
                   for k, f, col in (("max_dlnz", np.max, 0), ("median_dlnz", np.median, 0),
                                     ("max_dchi2_over_dense_min", np.max, 1),
                                     ("median_dchi2_over_dense_min", np.median, 1))})}


def adjoint_study(rtg, tms, torch):
    """Config 2: chi2, dchi2/dz, d2chi2/dz2 and dchi2/dflux (the adjoint pair
    kernel, rr_zscan_pairs_grad) for every target of the workload against
    every template at 3 redshifts each (as for the top 3 minima)."""
    from redrock_b200.adjoint import PairContext
    from redrock_b200.engine import pair_ranges_ok, run_pairs_grad
    rng = np.random.default_rng(5)
    npairs = 0
    ms = 0.0
    for tm in tms:
        ctx = PairContext(rtg, tm)
        z = np.asarray(tm.redshifts)
        pz = rng.choice(z[1:-1], size=3 * len(rtg))
        pt = np.repeat(np.arange(len(rtg)), 3).astype(np.int32)
        ok = pair_ranges_ok(ctx.src, ctx.layout, pz)
        pt, pz = pt[ok], pz[ok]
        run_pairs_grad(ctx.rows, ctx.src, pt, pz, want_dflux=True)   # warm-up
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        run_pairs_grad(ctx.rows, ctx.src, pt, pz, want_dflux=True)
        b.record()
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
        npairs += len(pz)
    return {"pairs": npairs, "ms": ms, "value": npairs / (ms / 1e3),
            "unit": "gradient evals/s (chi2, dchi2/dz, d2chi2/dz2, dchi2/dflux per (target, z))",
            "kernel": "zscan_pairs_kernel<NB, grad> (template rebinned + IGM per pair)"}


def archetype_study(tg, rtg, torch, narch=24):
    """Archetype refits (archetypes.py:295-400) of every target of the
    workload at its true redshift: per-camera fits with 2 Legendre terms per
    camera and prior sigma 0.1 against narch synthetic GALAXY archetypes,
    all targets in one best_archetypes call (rebin x IGM of every archetype
    at every redshift, then the rr_archetype_fit launches)."""
    from redrock_b200 import archetypes as A, fitz, synth
    arch = A.Archetype.from_synth(synth.archetype_set(narch=narch, seed=5))
    items = []
    for t, ts in zip(rtg, tg):
        t.legendre(2)
        items.append((t, ts.ztrue, None))
    prior = fitz.prior_on_coeffs(1, 2, 0.1, 3)
    arch.best_archetypes(items, True, None, prior=prior)   # warm-up
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    arch.best_archetypes(items, True, None, prior=prior)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    nfit = len(items) * narch
    return {"fits": nfit, "ms": ms, "value": nfit / (ms / 1e3),
            "unit": "archetype fits/s (one archetype + per-camera Legendre terms at one z)",
            "kernels": "arch_pair_kernel, arch_gram_kernel, arch_solve_kernel (+ rr_trapz_rebin)"}


def ygemm_study(args, step, torch, evals):
    """Throughput and zchi2/zcoeff error of each y variant (FP64 in the
    scan, or the tensor-core GEMM in bf16x3 / tf32x3 / int8x7 / int8x6), errors
    against the FP64 path on the same workload."""
    huge = 9999999.0
    out = {}
    ref = None
    fwf = None
    for v in ["fp64", "bf16x3", "tf32x3", "int8x7", "int8x6"]:
        step(False, ygemm=v)
        torch.cuda.synchronize()
        ev = []
        res, pack = step(True, ygemm=v, sink=ev)
        torch.cuda.synchronize()
        ms = ev[0][0].elapsed_time(ev[0][1])
        ent = {"value": evals / (ms / 1e3), "unit": "chi2 evals/s", "scan_ms": ms}
        if v == "fp64":
            ref = res
            rows = pack.rows.long()
            lane_fwf = pack.fwf
            fwf = torch.zeros(int(rows.max()) + 1, dtype=torch.float64, device=lane_fwf.device)
            ok = rows >= 0
            fwf[rows[ok]] = lane_fwf[ok]
        else:
            dmax, drel, agree, n, cmax = 0.0, 0.0, 0, 0, 0.0
            for a, b in zip(res, ref):
                good = b.zchi2 < huge
                d = (a.zchi2 - b.zchi2).abs().where(good, torch.zeros_like(b.zchi2))
                dmax = max(dmax, float(d.max()))
                drel = max(drel, float((d / fwf[:, None].clamp_min(1e-300)).max()))
                agree += int((a.zchi2.argmin(dim=1) == b.zchi2.argmin(dim=1)).sum())
                n += a.zchi2.shape[0]
                sc = b.zcoeff.abs().amax(dim=-1, keepdim=True).clamp_min(1e-300)
                cmax = max(cmax, float(((a.zcoeff - b.zcoeff).abs() / sc).max()))
            ent.update({"max_abs_dchi2": dmax, "max_dchi2_over_fTWf": drel,
                        "best_z_index_agreement": agree / n, "max_rel_dcoeff": cmax,
                        "meets_dchi2_1e-3": dmax <= 1e-3})
        out[v] = ent
        del res
    out["reference"] = ("errors against this engine's FP64 scan on the same workload "
                        "(itself within |dchi2| <= 2e-5 of the oracle in tests/)")
    return out


# ---------------------------------------------------------------------------
# CPU baseline: redrock's own CPU path (the unmodified install at
# baseline/_ref), or the oracle restatement when that install is absent
# ---------------------------------------------------------------------------
REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def reference_available():
    return os.path.exists(os.path.join(REF_DIR, "redrock", "zscan.py"))


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _import_reference():
    """redrock from baseline/_ref, unmodified.  astropy and fitsio are not
    installed; redrock uses them only for file I/O and zfind's output table,
    so empty stand-in modules satisfy its imports."""
    import types
    for name in ("astropy", "astropy.io", "astropy.io.fits", "astropy.table", "fitsio"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["astropy"].io = sys.modules["astropy.io"]
    sys.modules["astropy"].table = sys.modules["astropy.table"]
    sys.modules["astropy.io"].fits = sys.modules["astropy.io.fits"]
    sys.modules["astropy.io.fits"].open = None
    sys.modules["astropy.table"].Table = None
    sys.modules["fitsio"].FITS = None
    sys.path.insert(0, REF_DIR)
    import redrock.igm  # noqa: F401
    import redrock.rebin  # noqa: F401
    import redrock.targets  # noqa: F401
    import redrock.templates  # noqa: F401
    import redrock.zscan  # noqa: F401
    return sys.modules["redrock"]


def _reference_samples(workload, per_core, zsub, seed, ncores, nsample):
    """nsample samples of the workload through redrock's own CPU path, in
    this (torch-free) process: per sample, DistTemplate of every template
    on every zsub-th redshift (one process, as redrock does without MPI),
    then calc_zchi2_targets(mp_procs=ncores) over ncores * per_core
    targets.  Each sample is extrapolated to the whole workload: template
    builds scale with the redshifts per template, the scan with the
    evaluations."""
    import contextlib
    import io

    import scipy.sparse
    rr = _import_reference()
    from redrock_b200 import synth
    tr = None
    if "qso_frac" in WORKLOADS[workload]:
        def tr(z, w):
            return rr.igm.transmission_Lyman(np.array([z]), w, model="Inoue14")[0]
    full_nz = [len(ts.redshifts) for ts in synth.template_set()]
    tset = synth.template_set(zsub=zsub)
    # the rebin's numba JIT compiles before anything is timed
    rr.rebin.trapz_rebin(np.arange(10.), np.ones((1, 10)), edges=[1., 2., 3.],
                         myz=np.array([0.0]))
    ntarget_full = WORKLOADS[workload]["ntarget"]
    out = []
    for k in range(nsample):
        tg = synth_targets(workload, ncores * per_core, seed + k, transmission=tr)
        targets = []
        for t in tg:
            sp = [rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(),
                                      scipy.sparse.dia_matrix((s.rdata, s.roffsets),
                                                              shape=(len(s.wave),) * 2),
                                      band=s.band) for s in t.spectra]
            targets.append(rr.targets.Target(t.targetid, sp))
        tms = [rr.templates.Template(spectype=ts.spectype, subtype=ts.subtype,
                                     redshifts=ts.redshifts, wave=ts.wave, flux=ts.flux,
                                     method=ts.method, igm_model=ts.igm_model) for ts in tset]
        dtg = rr.targets.DistTargetsCopy(targets)
        dwave = dtg.wavegrids()
        build = []
        with contextlib.redirect_stdout(io.StringIO()):
            dts = []
            for tm in tms:
                t0 = time.perf_counter()
                dts.append(rr.templates.DistTemplate(tm, dwave))
                build.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            rr.zscan.calc_zchi2_targets(dtg, dts, mp_procs=ncores)
            scan = time.perf_counter() - t0
        evals = len(targets) * sum(len(ts.redshifts) for ts in tset)
        evals_full = ntarget_full * sum(full_nz)
        build_full = sum(b * nf / len(ts.redshifts) for b, nf, ts in zip(build, full_nz, tset))
        scan_full = scan * evals_full / evals
        out.append({"version": getattr(rr, "__version__", "unknown"),
                    "evals": evals, "build_s": sum(build), "scan_s": scan,
                    "value": evals_full / (build_full + scan_full),
                    "scan_value": evals / scan, "build_full_s": build_full,
                    "scan_full_s": scan_full, "targets": len(targets)})
    return out


def _cpu_worker(args):
    seed, ntarget, zsub, barrier = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from redrock_b200 import synth
    tg = synth.make_targets(ntarget, seed=seed)
    tset = synth.template_set(zsub=zsub)
    grids = synth.camera_grids()
    bases = []
    for ts in tset:
        bases.append((ts, O.template_basis(ts.wave, ts.flux, ts.redshifts, grids, ts.igm_model),
                      O.oii_template(ts.wave, ts.flux) if ts.spectype == "GALAXY" else None))
    ospec = [[O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
              for s in t.spectra] for t in tg]
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    evals = 0
    for ts, tdata, oii in bases:
        O.calc_zchi2(ospec, tdata, len(ts.redshifts), ts.flux.shape[0], OIItemplate=oii)
        evals += len(tg) * len(ts.redshifts)
    return evals, time.perf_counter() - t0


def port_scan_sample(nproc, per_worker, zsub, seed=1):
    """(evals/s, cores, sample description) of the oracle restatement of
    redrock's scan on host cores (bases built before timing)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        barrier = mgr.Barrier(nproc) if nproc > 1 else None
        with ctx.Pool(nproc) as pool:
            res = pool.map(_cpu_worker, [(seed + i, per_worker, zsub, barrier)
                                         for i in range(nproc)])
    evals = sum(r[0] for r in res)
    wall = max(r[1] for r in res)
    sample = (f"oracle restatement (redrock install absent): {nproc} processes x {per_worker} "
              f"targets x all 7 templates at every {zsub}th redshift ({evals} evals, "
              f"{wall:.1f} s); bases built before timing")
    return evals / wall, nproc, sample


def reference_cpu(workload, per_core, zsub, seed, nsample):
    """Samples of redrock's own CPU path, each run in a fresh interpreter
    (no CUDA context in the processes redrock forks).  Returns (samples,
    cores, description) or None when baseline/_ref is absent."""
    if not reference_available():
        return None
    ncores = host_cores()
    env = dict(os.environ)
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMBA_NUM_THREADS"):
        env[k] = "1"
    cmd = [sys.executable, os.path.abspath(__file__), "--reference-worker",
           json.dumps({"workload": workload, "per_core": per_core, "zsub": zsub, "seed": seed,
                       "ncores": ncores, "nsample": nsample})]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"reference worker failed: {r.stderr[-2000:]}")
    samples = json.loads(r.stdout.strip().splitlines()[-1])
    s0 = samples[-1]
    ver = s0["version"]
    desc = (f"redrock {ver} (unmodified, baseline/_ref) on {ncores} host cores: per sample "
            f"{s0['targets']} targets x 7 templates at every {zsub}th redshift "
            f"({s0['evals']} evals); DistTemplate builds {s0['build_s']:.2f} s (one process, "
            f"as redrock without MPI), calc_zchi2_targets(mp_procs={ncores}) "
            f"{s0['scan_s']:.2f} s; extrapolated to {WORKLOADS[workload]['ntarget']} targets on "
            f"the full z grids (builds x redshifts, scan x evals): "
            f"{s0['build_full_s']:.1f} s + {s0['scan_full_s']:.1f} s")
    return samples, ncores, desc


def cpu_baseline_entry(workload, args):
    """The cpu_baseline object of our arm's line (one bounded sample)."""
    ref = reference_cpu(workload, args.ref_per_core, args.ref_zsub, seed=100, nsample=1)
    if ref is not None:
        samples, cores, desc = ref
        return {"value": samples[0]["value"], "unit": "chi2 evals/s", "cores": cores,
                "kind": "reference", "sample": desc,
                "scan_only_value": samples[0]["scan_value"]}
    v, cores, sample = port_scan_sample(host_cores(), 4, 5)
    return {"value": v, "unit": "chi2 evals/s", "cores": cores, "kind": "port", "sample": sample}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    ref = reference_cpu(args.workload, args.ref_per_core, args.ref_step_zsub, seed=100,
                        nsample=args.warmup + args.steps)
    if ref is not None:
        samples, cores, desc = ref
        vals = [x["value"] for x in samples[args.warmup:]]
        kind = "reference"
    else:
        vals = []
        for i in range(args.warmup + args.steps):
            v, cores, desc = port_scan_sample(host_cores(), 4, 5, seed=100 + i)
            if i >= args.warmup:
                vals.append(v)
        kind = "port"
    value = float(np.median(vals))
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "chi2 evals/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded DESI-like targets and templates, redrock_b200/synth.py)",
        "config": {"workload": WORKLOAD_NAMES[args.workload]},
        "cpu_baseline": {"value": value, "unit": "chi2 evals/s", "cores": cores, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": "chi2 evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--ntargets", type=int, default=None,
                    help="override the workload's number of targets")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--zsub", type=int, default=None,
                    help="keep every zsub-th redshift (small profiling cases only)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=8,
                    help="end-to-end steps timed (at most --steps)")
    ap.add_argument("--ygemm", default=None,
                    choices=["fp64", "bf16x3", "tf32x3", "int8x7", "int8x6"],
                    help="y = Tb^T W f as a tensor-core GEMM (int8x7 / int8x6: exact; the "
                         "engine's default when not given) or summed in the FP64 scan (fp64)")
    ap.add_argument("--archetypes", action="store_true",
                    help="also time batched archetype refits of every target (24 archetypes)")
    ap.add_argument("--adjoint", action="store_true",
                    help="also time the adjoint pair kernel on 3 redshifts per target and template")
    ap.add_argument("--zfind", action="store_true",
                    help="also time zfind (eager, CUDA graph, Newton) on --zfind-targets targets "
                         "and check the refined redshifts against dense FP64 scans")
    ap.add_argument("--zfind-targets", type=int, default=500,
                    help="targets of the workload the zfind study uses (default 500)")
    ap.add_argument("--tiles", default=None,
                    help='fixed tile choice as JSON, e.g. \'{"4": 3, "5": 2, "block_group": 4}\' '
                         "(skips the autotuner)")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="use the default tile shapes instead of timing them before the run")
    ap.add_argument("--ygemm-study", action="store_true",
                    help="also time every y variant once and report its chi2/coeff error")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the desi500 line reported beside the main workload")
    ap.add_argument("--no-graph", dest="graph", action="store_false",
                    help="launch every step eagerly instead of replaying the step as one "
                         "captured CUDA graph")
    ap.add_argument("--plain-targets", type=int, default=8)
    ap.add_argument("--ref-zsub", type=int, default=10,
                    help="redshift subsampling of the cpu_baseline sample")
    ap.add_argument("--ref-step-zsub", type=int, default=10,
                    help="redshift subsampling of each --impl reference step")
    ap.add_argument("--ref-per-core", type=int, default=2,
                    help="targets per host core in a reference sample")
    ap.add_argument("--reference-worker", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.reference_worker is not None:
        # child process of reference_cpu: redrock's CPU path, no torch
        kw = json.loads(args.reference_worker)
        print(json.dumps(_reference_samples(**kw)))
        return
    rank, world, local_rank = env_rank()
    if args.impl == "reference":
        # rank 0 alone times the CPU path; the other ranks have no work
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = run_ours(args, rank, world, local_rank)
    if out is not None and world == 1 and not args.no_extra and args.workload != "desi500" \
            and not args.ntargets and not args.zsub:
        # the 500-target batch beside the main workload (fewer steps)
        ex = argparse.Namespace(**vars(args))
        ex.workload = "desi500"
        ex.steps, ex.warmup = min(args.steps, 5), min(args.warmup, 3)
        ex.e2e_steps = min(args.e2e_steps, 5)
        ex.no_plain = False
        ex.plain_targets = args.plain_targets
        ex.ygemm_study = ex.adjoint = ex.archetypes = False
        import torch
        torch.cuda.empty_cache()
        d = run_ours(ex, rank, world, local_rank)
        out["desi500"] = {k: d[k] for k in ("value", "ms_per_step", "e2e", "plain", "roofline",
                                            "config", "clocks", "gpu_launches")}
    if out is not None and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_entry(args.workload, args)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
