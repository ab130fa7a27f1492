#!/usr/bin/env python
"""Benchmark of the B200 plane-wave FGT on its headline workload.

Metric: FGT points/s at eps = 1e-6 (the mixed form; the FP64 plain form is
timed beside it on the same GPU, key ``fp64_form``).  Workload (default): the 2D strongly clustered
adaptive-tree case -- N = 1e7 sources = targets, 90% on a circle of radius 0.3
about (0.5, 0.5) with Gaussian radial jitter sigma = 1e-3, 10% uniform in the
unit square, charges N(0,1), delta = 1e-6, eps = 1e-6, potential at the
sources (ifpgh = 1, ifpghtarg = 0); seeded synthetic data.

points/s = (ns + targets evaluated) / time.  ``value`` times one execute of a
prebuilt plan with inputs resident in HBM (gather -> form -> merge -> mp->loc
-> split -> eval -> near field -> scatter); ``e2e`` times the drop-in call
(host tree and lists, host->device copies from pinned memory, transform,
device->host copy of the potentials).  ``errors`` gives the relative l2 error
(the reference driver's ``derr``) of the timed outputs against an FP64 direct
sum at 1e4 sampled points and against the oracle on the whole workload.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--workload cfg2|cfg1|cfg3|cfg4_d1e-2_e1e-6|...]
Multi-GPU (N > 1, torchrun): independent replicas, one per rank.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


# ------------------------------------------------------------------ workloads
def make_workload(name: str, seed: int):
    rng = np.random.default_rng(seed)
    if name in ("cfg2", "cfg2_n2e6"):
        n = 10_000_000 if name == "cfg2" else 2_000_000
        m = int(0.9 * n)
        th = rng.random(m) * 2 * np.pi
        r = 0.3 + rng.normal(0.0, 1e-3, m)
        p = np.empty((n, 2))
        p[:m, 0] = 0.5 + r * np.cos(th)
        p[:m, 1] = 0.5 + r * np.sin(th)
        p[m:] = rng.random((n - m, 2))
        q = rng.standard_normal(n)
        return dict(name=f"2d_circle_clustered_N{n:.0e}_d1e-6_e1e-6".replace("+0", ""), dim=2, nd=1, delta=1e-6, eps=1e-6,
                    src=p, chg=q, trg=p, ifpgh=1, ifpghtarg=0)
    if name == "cfg1":
        n = 100_000
        return dict(name="2d_uniform_N1e5+1e5_d1e-4_e1e-9", dim=2, nd=1, delta=1e-4, eps=1e-9,
                    src=rng.random((n, 2)), chg=rng.random(n), trg=rng.random((n, 2)), ifpgh=1,
                    ifpghtarg=1)
    if name in ("cfg3", "cfg3_n5e5"):
        n = 4_000_000 if name == "cfg3" else 500_000
        c = rng.random((16, 3)) * 0.8 + 0.1

        def pts(k):
            lab = rng.integers(0, 16, k)
            x = c[lab] + rng.normal(0, 0.02, (k, 3))
            u = rng.random(k) < 0.2
            x[u] = rng.random((int(u.sum()), 3))
            return x

        return dict(name=f"3d_blobs_N{n:.0e}+{n:.0e}_d1e-3_e1e-6".replace("+0", ""), dim=3, nd=1, delta=1e-3, eps=1e-6,
                    src=pts(n), chg=2 * rng.random(n) - 1, trg=pts(n), ifpgh=0, ifpghtarg=1)
    if name.startswith("cfg4"):
        _, d, e = name.split("_")
        n = 2_000_000
        x = rng.random((n, 3))
        return dict(name=f"3d_uniform_N2e6_{d}_{e}", dim=3, nd=1, delta=float(d[1:]),
                    eps=float(e[1:]), src=x, chg=rng.random(n), trg=x, ifpgh=1, ifpghtarg=0)
    raise SystemExit(f"unknown workload {name}")


def points_of(w):
    return w["src"].shape[0] * (1 if w["ifpgh"] else 0) + (w["trg"].shape[0] if w["ifpghtarg"] else 0)


# DRAM bytes (read + write) of one launch of the dominant kernel, from the
# committed ncu capture named beside each figure
PROFILED_TRAFFIC = {
    ("2d_circle_clustered_N1e7_d1e-6_e1e-6", "k_form2d_mma<2>"):
        (216619776 + 16602112, "profiles/form2d_mma_2d_circle_N1e7.md"),
}
# The same from a capture of a smaller case of the same distribution, delta
# and eps (so the same orders): DRAM bytes of the captured launch and its
# executed flops; a launch's traffic is scaled by its executed flops (the
# kernel reads each of its sources once, so traffic grows with them).
PROFILED_TRAFFIC_SCALED = {
    ("k_form2d_f32", 1e-6, 1e-6): (43087872 + 176384, 596234028.0,
                                   "profiles/form2d_f32_2d_circle_N2e6.md (N = 2e6 capture, scaled by "
                                   "the launch's executed flops)"),
}


# ------------------------------------------------------------------ clocks
_REASON_BITS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
                0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every ~1 ms in a
    background thread while the timed loop runs (the timed region of a short
    run lasts only tens of ms, too short for nvidia-smi's 200 ms polling).
    Falls back to nvidia-smi polling when NVML is not importable."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.sm: list[float] = []
        self.reasons: set[str] = set()
        self.smax = None
        self.proc = None
        self.lines: list[str] = []
        self.stop_ev = threading.Event()
        self.nv = None
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = None
            try:
                import torch
                pr = torch.cuda.get_device_properties(device)
                h = nv.nvmlDeviceGetHandleByUUID("GPU-" + str(pr.uuid))
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(device)
            self.nv, self.h = nv, h
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._sample()
            self.t = threading.Thread(target=self._loop, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _sample(self):
        nv, h = self.nv, self.h
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
        try:
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        for bit, name in _REASON_BITS.items():
            if r & bit:
                self.reasons.add(name)

    def _loop(self):
        while not self.stop_ev.wait(0.001):
            try:
                self._sample()
            except Exception:
                break

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nv is not None:
            self.stop_ev.set()
            self.t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                    "sm_max_mhz": self.smax, "reasons": sorted(self.reasons),
                    "samples": len(self.sm), "source": "nvml, 1 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ------------------------------------------------------------------ helpers
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


METRIC = "FGT points/s at eps 1e-6"
N_ERR_SAMPLE = 10_000  # targets of the sampled-target error against the FP64 direct sum


def config_of(w):
    """The workload's config object, identical in both arms."""
    return {"workload": w["name"], "dim": w["dim"], "points_per_step": points_of(w),
            "ns": int(w["src"].shape[0]), "nt": int(w["trg"].shape[0]), "delta": w["delta"],
            "eps": w["eps"], "ifpgh": w["ifpgh"], "ifpghtarg": w["ifpghtarg"],
            "l2": "inputs larger than the 126 MB L2 (no flush)"}


def slab_sample(w, frac=1.0 / 16):
    """The points with x below the `frac` quantile of the sources' x: a
    spatially contiguous piece of the workload.  Unlike a random subset it
    keeps the local density (near-field pairs per point, leaf sizes) and the
    root box size (set by the largest extent), so its per-point cost stands
    for the whole workload's."""
    xs = w["src"][:, 0]
    a = float(np.quantile(xs, frac))
    si = xs < a
    out = dict(w)
    out["src"], out["chg"] = w["src"][si], w["chg"][si]
    out["trg"] = out["src"] if w["trg"] is w["src"] else w["trg"][w["trg"][:, 0] < a]
    out["slab_x"] = a
    return out


def run_oracle(w, nthreads):
    """One oracle transform of workload `w`: (points, seconds, pot, pottarg)."""
    from oracle import oracle as O
    O.build()
    t0 = time.perf_counter()
    pot, pt, _ = O.fgt(w["dim"], w["nd"], w["delta"], w["eps"], w["src"], w["chg"], w["trg"],
                       w["ifpgh"], w["ifpghtarg"], nthreads=nthreads)
    dt = time.perf_counter() - t0
    return points_of(w), dt, pot, pt


def error_sample(w, seed=99):
    """Sampled evaluation points (1e4, or all when fewer) with the FP64
    direct sum at them: (which, idx, exact), which = "pot" or "pottarg"."""
    from oracle import oracle as O
    O.build()
    rng = np.random.default_rng(seed)
    if w["ifpghtarg"]:
        which, pts = "pottarg", w["trg"]
    else:
        which, pts = "pot", w["src"]
    idx = np.sort(rng.choice(pts.shape[0], min(N_ERR_SAMPLE, pts.shape[0]), replace=False))
    exact = O.direct_cut(w["dim"], w["nd"], w["delta"], w["src"], w["chg"].reshape(-1, w["nd"]),
                         pts[idx])
    return which, idx, exact


def derr(a, b):
    from oracle import oracle as O
    return float(O.derr(a, b))


# ------------------------------------------------------------------ arms
def reference_arm(args, w, rank, world):
    """The reference's CPU path (the oracle port: no Fortran compiler exists on
    either machine, so the reference itself cannot be built) on the full
    workload, all host threads, one transform per step."""
    if rank != 0:
        return 0
    cores = cpu_cores()
    for i in range(args.warmup):
        run_oracle(w, cores)
    times, pts = [], 0
    for i in range(args.steps):
        p, dt, _, _ = run_oracle(w, cores)
        times.append(dt)
        pts = p
    ms = 1e3 * sum(times) / len(times)
    v = pts / (ms / 1e3)
    one = single_thread_baseline(w) if not args.no_cpu_baseline else None
    line = {"impl": "reference", "metric": METRIC, "value": v,
            "unit": "points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded numpy)",
            "config": config_of(w),
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "port",
                             "sample": f"the full workload each step ({w['src'].shape[0]} sources), "
                                       f"oracle (C++ restatement of the reference) on {cores} threads",
                             "single_thread": one},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def single_thread_baseline(w):
    """The oracle on one thread (the reference's default build, OMP=OFF) over
    a contiguous slab holding 1/16 of the points, so the run takes seconds."""
    sw = slab_sample(w)
    p, dt, _, _ = run_oracle(sw, 1)
    return {"value": p / dt, "unit": "points/s", "cores": 1, "kind": "port", "seconds": dt,
            "sample": f"slab x < {sw['slab_x']:.4f} of the workload ({sw['src'].shape[0]} sources, "
                      f"{p} points evaluated): same local density and root box as the full run"}


def ours_arm(args, w, rank, world, local_rank):
    import torch
    import fgt2d_b200 as F

    dev = local_rank
    torch.cuda.set_device(dev)
    pts = points_of(w)
    dim, nd = w["dim"], w["nd"]

    # plan (tree + lists + device tasks), built once; the context's precision
    # selects the form at each execute
    ctx = F.Context(dev, precision="mixed", scheme=args.scheme)
    t0 = time.perf_counter()
    plan = F.Plan(ctx, dim, nd, w["delta"], w["eps"], w["src"], w["trg"], w["ifpgh"],
                  w["ifpghtarg"])
    plan_s = time.perf_counter() - t0
    info = plan.info()
    d_src = torch.from_numpy(np.ascontiguousarray(w["src"])).to(f"cuda:{dev}")
    d_chg = torch.from_numpy(np.ascontiguousarray(w["chg"]).reshape(-1, nd)).to(f"cuda:{dev}")
    d_trg = d_src if w["trg"] is w["src"] else torch.from_numpy(np.ascontiguousarray(w["trg"])).to(f"cuda:{dev}")
    d_pot = torch.zeros((w["src"].shape[0], nd), dtype=torch.float64, device=f"cuda:{dev}")
    d_pt = torch.zeros((w["trg"].shape[0], nd), dtype=torch.float64, device=f"cuda:{dev}")
    # a dedicated stream: the plan's kernels and the timing events share it
    stream = torch.cuda.Stream(dev)
    sp = stream.cuda_stream

    def step(precision):
        ctx.set_precision(precision)
        plan.execute_device(d_src.data_ptr(), d_chg.data_ptr(), d_trg.data_ptr(),
                            d_pot.data_ptr(), d_pt.data_ptr(), stream=sp)

    from fgt2d_b200.replicas import barrier, max_over_ranks

    results, outputs = {}, {}
    clocks = None
    for prec in ("fp64", "mixed"):  # mixed last: its clocks are the headline's
        for _ in range(args.warmup):
            step(prec)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        sampler = ClockSampler(dev) if prec == "mixed" else None
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step(prec)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        if sampler is not None:
            clocks = sampler.stop()
        ms = e0.elapsed_time(e1) / args.steps
        results[prec] = max_over_ranks(ms)
        # the last timed step's outputs, for the errors below
        outputs[prec] = (d_pot.cpu().numpy().copy() if w["ifpgh"] else None,
                         d_pt.cpu().numpy().copy() if w["ifpghtarg"] else None)
    # per-stage device times (CUDA events around each stage, on the plan's
    # stream) over K further steps of each precision
    stages = {}
    for prec in ("fp64", "mixed"):
        ctx.set_precision(prec)
        acc = {}
        for _ in range(args.steps):
            s = plan.profile_device(d_src.data_ptr(), d_chg.data_ptr(), d_trg.data_ptr(),
                                    d_pot.data_ptr(), d_pt.data_ptr())
            for k, v in s.items():
                acc[k] = acc.get(k, 0.0) + v / args.steps
        stages[prec] = acc
    stage = stages["mixed"]
    launches_per_step = plan.info()["kernel_launches"]

    # end to end through the public API from pinned host memory
    src_h = torch.from_numpy(np.ascontiguousarray(w["src"])).pin_memory().numpy()
    chg_h = torch.from_numpy(np.ascontiguousarray(w["chg"]).reshape(-1, nd)).pin_memory().numpy()
    trg_h = src_h if w["trg"] is w["src"] else torch.from_numpy(np.ascontiguousarray(w["trg"])).pin_memory().numpy()
    # the results land in pinned host buffers (allocated once, outside the timing)
    out_h = {}
    if w["ifpgh"]:
        out_h["pot"] = torch.zeros((w["src"].shape[0], nd), dtype=torch.float64).pin_memory().numpy()
    if w["ifpghtarg"]:
        out_h["pottarg"] = torch.zeros((w["trg"].shape[0], nd), dtype=torch.float64).pin_memory().numpy()
    e2e_steps = 0 if args.no_e2e else max(1, min(args.steps, 5))
    ctx.set_precision("mixed")
    e2e_s = float("nan")
    if e2e_steps:
        F.transform(dim, nd, w["delta"], w["eps"], src_h, chg_h, trg_h, w["ifpgh"], w["ifpghtarg"],
                    ctx=ctx, out=out_h)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            F.transform(dim, nd, w["delta"], w["eps"], src_h, chg_h, trg_h, w["ifpgh"],
                        w["ifpghtarg"], ctx=ctx, out=out_h)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
    h2d = src_h.nbytes + chg_h.nbytes + (trg_h.nbytes if w["ifpghtarg"] else 0)
    d2h = (w["src"].shape[0] * nd * 8 if w["ifpgh"] else 0) + (w["trg"].shape[0] * nd * 8 if w["ifpghtarg"] else 0)

    if rank != 0:
        return 0
    hbm, tf, peak_src = measured_peaks()
    fp64_tf = ctx.fp64_mma_tflops()
    # roofline of the dominant tensor-core launch (the Hermite-block kernel of
    # the form order group with the most sources), timed with CUDA events
    # around that launch alone over K further executes on the plan's stream
    ctx.set_precision("mixed")
    dms, dfl, dalg, dname = [], 0.0, 0.0, None
    for _ in range(args.steps):
        r = plan.profile_dominant(d_chg.data_ptr(), d_pot.data_ptr(), d_pt.data_ptr())
        if r is None:
            break
        dms.append(r[0])
        dfl, dname, dalg = r[1], r[2], r[3]
    if dms:
        t_k = sum(dms) / len(dms) / 1e3
        ach = dalg / t_k / 1e12
        traffic, tsrc = PROFILED_TRAFFIC.get((w["name"], dname), (None, None))
        sc = PROFILED_TRAFFIC_SCALED.get((dname, w["delta"], w["eps"]))
        if traffic is None and sc is not None and dfl > 0:
            traffic, tsrc = sc[0] * dfl / sc[1], sc[2]
        roof = {"bound": "tensor", "kernel": dname, "stage": "form", "achieved": ach, "peak": tf,
                "unit": "TFLOP/s", "frac": ach / tf, "traffic": traffic,
                "peak_source": f"{peak_src} bf16 dense (burst), MEASURED_PEAKS.json",
                "work": f"{dalg:.4g} algorithmic flops per launch = 4 n npw^d nd over the "
                        f"launch's n sources (plane-wave form count)",
                "launch_ms": t_k * 1e3,
                "executed_flops": dfl, "executed_tflops": dfl / t_k / 1e12,
                "fp64_mma_peak_probe_tflops": fp64_tf,
                "executed_frac_of_fp64_mma": dfl / t_k / 1e12 / fp64_tf}
        if tsrc:
            roof["traffic_source"] = tsrc
    else:
        roof = {"bound": "tensor", "kernel": None, "achieved": None, "peak": tf, "unit": "TFLOP/s",
                "frac": None, "traffic": None, "note": "no tensor-core launch in this plan"}
    sb = info["shift_bytes"]
    t_b = (stage.get("merge", 0) + stage.get("m2l", 0) + stage.get("split", 0)) / 1e3
    roof_b = None
    if t_b > 0:
        gbs = (sb[0] + sb[1] + sb[2]) / t_b / 1e9
        roof_b = {"bound": "hbm", "stage": "shifts (merge + mp->loc + split)", "achieved": gbs,
                  "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                  "work": f"{sb[0] + sb[1] + sb[2]:.4g} bytes per step: 16 B per complex "
                          f"coefficient, each distinct expansion read or written once per stage",
                  "stage_ms": t_b * 1e3}
    stage_rates = {
        "form_tflops_algorithmic": info["form_flops"] / (stage["form"] / 1e3) / 1e12 if stage.get("form") else None,
        "eval_tflops_algorithmic": info["eval_flops"] / (stage["eval"] / 1e3) / 1e12 if stage.get("eval") else None,
        "form_tflops_executed": info["form_route_flops"] / (stage["form"] / 1e3) / 1e12 if stage.get("form") else None,
        "eval_tflops_executed": info["eval_route_flops"] / (stage["eval"] / 1e3) / 1e12 if stage.get("eval") else None,
        "direct_pairs_per_s": info["direct_pairs"] / (stage["direct"] / 1e3) if stage.get("direct") else None,
        "fp64_mma_peak_probe_tflops": fp64_tf,
    }
    # errors of the timed outputs: FP64 direct sum at 1e4 sampled points, and
    # the oracle (restated reference) on the whole workload
    errors = None
    cpu_base = None
    if not args.no_errors:
        which, idx, exact = error_sample(w)
        k = 0 if which == "pot" else 1
        errors = {"metric": "derr (relative l2, test_fgt2d.f:204-225)",
                  "direct_sample": f"FP64 direct sum (pairs within sqrt(delta ln 1e30)) at {idx.size} "
                                   f"sampled {'sources' if k == 0 else 'targets'}",
                  "err_vs_direct": derr(exact, outputs["mixed"][k][idx]),
                  "err_vs_direct_fp64": derr(exact, outputs["fp64"][k][idx])}
    if world == 1 and not args.no_cpu_baseline:
        cores = cpu_cores()
        p_cpu, dt_cpu, opot, opt = run_oracle(w, cores)
        cpu_base = {"value": p_cpu / dt_cpu, "unit": "points/s", "cores": cores, "kind": "port",
                    "sample": f"the full workload once ({w['src'].shape[0]} sources), oracle (C++ "
                              f"restatement of the reference plane-wave FGT) on {cores} threads, "
                              f"{dt_cpu:.1f} s",
                    "single_thread": single_thread_baseline(w)}
        if errors is not None:
            o = (opot, opt)
            k = 0 if w["ifpgh"] else 1
            errors["err_vs_oracle"] = derr(o[k], outputs["mixed"][k])
            errors["err_vs_oracle_fp64"] = derr(o[k], outputs["fp64"][k])
            errors["oracle_vs_direct"] = derr(exact, o[0 if which == "pot" else 1][idx])
    secondary = None
    if world == 1 and args.workload == "cfg2" and not args.no_secondary:
        # free the headline plan's device memory first
        plan.close()
        del d_src, d_chg, d_trg, d_pot, d_pt
        torch.cuda.empty_cache()
        secondary = secondary_workload("cfg3", dev, max(3, min(args.steps, 5)), 3, args.scheme)
    ms_mixed, ms_fp64 = results["mixed"], results["fp64"]
    line = {
        "metric": METRIC,
        "value": world * pts / (ms_mixed / 1e3),
        "unit": "points/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 + f32 (mixed form)", "form": "mixed",
        "data": "synthetic (seeded numpy)",
        "config": config_of(w),
        "parallelism": "replicas" if world > 1 else "single GPU",
        "fp64_form": {"value": world * pts / (ms_fp64 / 1e3), "ms_per_step": ms_fp64,
                      "mixed_over_fp64": ms_fp64 / ms_mixed},
        "errors": errors,
        "stages_ms": stage,
        "stages_ms_fp64": stages["fp64"],
        "plan": {k: info[k] for k in ("npwlevel", "nlevels", "nboxes", "npw", "nexp", "nform",
                                      "neval", "ndirect_tasks", "direct_pairs", "device_bytes")},
        "host_plan_s": plan_s,
        "e2e": {"value": world * pts / e2e_s, "unit": "points/s", "s_per_step": e2e_s,
                "steps": e2e_steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "includes": "tree build (point work on the GPU) + lists + plan upload + H2D from pinned inputs + transform + D2H into pinned outputs"},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": roof,
        "roofline_shifts": roof_b,
        "stage_rates": stage_rates,
        "cpu_baseline": cpu_base,
        "clocks": clocks,
        "secondary": secondary,
        "scheme": args.scheme,
    }
    print(json.dumps(line), flush=True)
    return 0


def secondary_workload(name, dev, steps, warmup, scheme="planewave"):
    """Device time of both forms on a second workload (the 3D blobs case by
    default) with inputs in HBM, per-stage times and the error of the timed
    outputs against the FP64 direct sum at 1e4 sampled points: reported
    beside the headline in the same line."""
    import torch
    import fgt2d_b200 as F
    w = make_workload(name, 1234 + 2)
    nd = w["nd"]
    ctx = F.Context(dev, precision="mixed", scheme=scheme)
    plan = F.Plan(ctx, w["dim"], nd, w["delta"], w["eps"], w["src"], w["trg"], w["ifpgh"], w["ifpghtarg"])
    d_src = torch.from_numpy(np.ascontiguousarray(w["src"])).to(f"cuda:{dev}")
    d_chg = torch.from_numpy(np.ascontiguousarray(w["chg"]).reshape(-1, nd)).to(f"cuda:{dev}")
    d_trg = d_src if w["trg"] is w["src"] else torch.from_numpy(np.ascontiguousarray(w["trg"])).to(f"cuda:{dev}")
    d_pot = torch.zeros((w["src"].shape[0], nd), dtype=torch.float64, device=f"cuda:{dev}")
    d_pt = torch.zeros((w["trg"].shape[0], nd), dtype=torch.float64, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(dev)
    out, outs, stages = {}, {}, {}
    for prec in ("fp64", "mixed"):
        ctx.set_precision(prec)
        run = lambda: plan.execute_device(d_src.data_ptr(), d_chg.data_ptr(), d_trg.data_ptr(),
                                          d_pot.data_ptr(), d_pt.data_ptr(), stream=stream.cuda_stream)
        for _ in range(warmup):
            run()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            run()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        out[prec] = e0.elapsed_time(e1) / steps
        outs[prec] = (d_pot.cpu().numpy().copy(), d_pt.cpu().numpy().copy())
        acc = {}
        for _ in range(steps):
            s = plan.profile_device(d_src.data_ptr(), d_chg.data_ptr(), d_trg.data_ptr(), d_pot.data_ptr(),
                                    d_pt.data_ptr())
            for k2, v in s.items():
                acc[k2] = acc.get(k2, 0.0) + v / steps
        stages[prec] = acc
    which, idx, exact = error_sample(w)
    k = 0 if which == "pot" else 1
    pts = points_of(w)
    res = {"workload": w["name"], "points_per_step": pts,
           "ms_per_step": out["mixed"], "value": pts / (out["mixed"] / 1e3),
           "fp64_ms_per_step": out["fp64"], "fp64_value": pts / (out["fp64"] / 1e3),
           "mixed_over_fp64": out["fp64"] / out["mixed"],
           "err_vs_direct": derr(exact, outs["mixed"][k][idx]),
           "err_vs_direct_fp64": derr(exact, outs["fp64"][k][idx]),
           "stages_ms": stages["mixed"], "stages_ms_fp64": stages["fp64"]}
    plan.close()
    return res


def serving_arm(args):
    """Serving stream: Poisson arrivals of transforms with mixed dimension, N,
    delta and eps, submitted to the transform server at their arrival times;
    latency is submit -> result on the host.  One base array of uniform
    points (and charges) is sliced for every request, so no generation time
    falls inside the arrival loop."""
    import threading as th

    import fgt2d_b200 as F

    n_req = args.requests
    rate = args.rate
    rng = np.random.default_rng(1234 + 5)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    dims = rng.integers(2, 4, n_req)
    ns = np.floor(10 ** rng.uniform(3, 6, n_req)).astype(int)
    deltas = 10 ** rng.uniform(-6, -1, n_req)
    epss = rng.choice([1e-3, 1e-6, 1e-9], n_req)
    nmax = int(ns.max())
    base = {2: rng.random((nmax, 2)), 3: rng.random((nmax, 3))}
    chg = rng.random(nmax)
    srv = F.Server(0, max_bytes=args.server_bytes, workers=args.workers, precision="auto",
                   sm_budget=args.server_sm_budget, grid_yield=args.server_grid_yield)
    # warm-up: one small request of each dimension (module load, first launches)
    for d in (2, 3):
        srv.wait(srv.submit(d, 1, 1e-3, 1e-6, base[d][:2000], chg[:2000]))
    ids = [None] * n_req
    lat = np.full(n_req, np.nan)
    status = np.zeros(n_req, dtype=int)
    done = th.Event()

    def waiter():
        for k in range(n_req):
            while ids[k] is None:
                time.sleep(1e-4)
            try:
                _, _, lat[k] = srv.wait(ids[k])
            except F.FGTError as e:
                status[k] = e.status
        done.set()

    wt = th.Thread(target=waiter, daemon=True)
    wt.start()
    t0 = time.perf_counter()
    for k in range(n_req):
        dt = arrivals[k] - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        d, n = int(dims[k]), int(ns[k])
        ids[k] = srv.submit(d, 1, float(deltas[k]), float(epss[k]), base[d][:n], chg[:n])
    done.wait()
    span = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    ok = status == 0
    small = ok & (ns <= 100_000)
    q = lambda a, f: float(np.quantile(a, f) * 1e3) if a.size else None
    pts = int(ns[ok].sum())
    line = {
        "metric": "serving p99 latency, requests with N <= 1e5", "value": q(lat[small], 0.99),
        "unit": "ms", "higher_is_better": False, "n_gpus": 1, "impl": "ours",
        "p50_ms_small": q(lat[small], 0.50), "p50_ms_all": q(lat[ok], 0.50), "p99_ms_all": q(lat[ok], 0.99),
        "max_ms_all": q(lat[ok], 1.0), "requests": n_req, "completed": int(ok.sum()),
        "failed": int((~ok).sum()),
        "failures": [[int(k), int(status[k]), int(dims[k]), int(ns[k]), float(deltas[k]), float(epss[k])]
                     for k in np.flatnonzero(~ok)[:8]],
        "points_per_s": pts / span, "span_s": span,
        "arrival_rate_per_s": rate, "workers": args.workers, "sm_budget": args.server_sm_budget, "grid_yield": args.server_grid_yield,
        "peak_device_bytes": st["peak_bytes"],
        "budget_device_bytes": st["budget_bytes"], "data": "synthetic (seeded numpy)",
        "config": {"workload": "serving stream: Poisson arrivals, dim in {2,3}, N log-uniform [1e3,1e6] "
                               "(sources = targets, uniform), charges U[0,1), delta log-uniform [1e-6,1e-1], "
                               "eps in {1e-3,1e-6,1e-9}", "ifpgh": 1, "ifpghtarg": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-errors", action="store_true", help="skip the sampled direct-sum errors")
    ap.add_argument("--no-secondary", action="store_true", help="skip the 3D blobs line beside the headline")
    ap.add_argument("--scheme", default="planewave", choices=["planewave", "nufft"],
                    help="algorithm of the timed plans: the plane-wave scheme (default) or the NUFFT scheme")
    ap.add_argument("--requests", type=int, default=4096, help="serving workload: number of requests")
    ap.add_argument("--rate", type=float, default=2000.0, help="serving workload: arrivals per second")
    ap.add_argument("--workers", type=int, default=8, help="serving workload: server worker streams")
    ap.add_argument("--server-bytes", type=int, default=0, help="serving workload: device budget (0: 80%% free)")
    ap.add_argument("--server-sm-budget", type=int, default=0,
                    help="serving workload: SMs a request's persistent kernels use (0: all)")
    ap.add_argument("--server-grid-yield", action="store_true",
                    help="serving workload: one CTA per task instead of persistent CTAs")
    args = ap.parse_args()
    if args.workload == "serving":
        return serving_arm(args)
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    from fgt2d_b200.replicas import replica_seed
    w = make_workload(args.workload, seed=replica_seed(1234 + 2, rank))
    if args.impl == "reference":
        return reference_arm(args, w, rank, world)
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            return ours_arm(args, w, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    return ours_arm(args, w, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
