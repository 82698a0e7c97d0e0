"""Benchmark of the residual path: Mcell-updates/s per RK stage, mixed vs FP64.

Workload (default): the 3D viscous frozen-chemistry periodic box, 128^3
points on a 2 mm cube, 9 species (synthetic data set in the reference's
ChemData format), Fourier-mode T/p/Y fields with a Taylor-Green velocity,
SSP-RK3 at CFL 0.5.  One step = 3 RK stages; value = points x 3 x steps /
time (summed over ranks).  Inputs stay resident in HBM; the working set
(~1.8 GB mixed) is far larger than the 126 MB L2, so no flush is needed.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU implementation of the path on the
host cores: the reference itself has no CPU path and its CUDA kernels cannot
be installed as a package, so the arm runs the C restatement of the
reference's algorithm (oracle/cc_oracle.c, pinned to the reference kernels by
tests/golden) with every host thread, on a bounded sample of the workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "box128_9sp_viscous_rk3"
E_STEPS = 1000  # steps of the workload's job (the end-to-end leg runs the whole job)
METRIC = "Mcell-updates/s per RK stage, mixed vs FP64 plain, at stated L2 err vs FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--err-steps", type=int, default=1000, help="steps of the mixed-vs-FP64 error check")
    ap.add_argument("--workload", default="box128",
                    choices=["box128", "multiblock64", "mixing_layer", "box256_closure", "box128_lusgs"],
                    help="box128: the headline 128^3 box; multiblock64: 64 uneven blocks, batched vs "
                         "per-block; mixing_layer: 1024x512x4 precision study (FP64 / mixed / FP32); "
                         "box256_closure: 256^3 box, exact transport vs the learned closure; "
                         "box128_lusgs: LU-SGS steady steps on the 128^3 box")
    ap.add_argument("--study-steps", default="100,1000,2000", help="mixing_layer: error snapshot steps")
    ap.add_argument("--variant", default="auto",
                    choices=["auto", "l1", "tma", "split", "split-tma", "split-tma-p", "dq-tma"],
                    help="stage kernels: autotuned (default) or pinned (profiling runs, where the autotuner's "
                         "timings are distorted)")
    ap.add_argument("--kz", type=int, default=4, help="k-planes per tile when --variant pins the stage kernels")
    ap.add_argument("--tile-j", type=int, default=0, help="points along j of the dq-tma tile when --variant pins it")
    ap.add_argument("--ref-n", type=int, default=128, help="box size of the reference-kernel timing (0 skips it)")
    ap.add_argument("--e2e-steps", type=int, default=E_STEPS, help="steps of the end-to-end job (profiling runs "
                                                                     "shorten it)")
    ap.add_argument("--ref-steps", type=int, default=2, help="timed steps of the reference-kernel timing")
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.
    The GPU is named by its UUID (the CUDA index and nvidia-smi's differ
    under CUDA_VISIBLE_DEVICES).  Entering waits for nvidia-smi's first
    sample, so the timed region starts with the sampler running; only the
    samples after that count.  A region shorter than the 50 ms interval
    takes the first sample after it."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.start = 0

    @staticmethod
    def _smi_id(index):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            return ids[index] if index < len(ids) else str(index)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self._smi_id(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 10:
                time.sleep(0.005)
        except Exception:
            self.proc = None
        self.start = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            t0 = time.time()
            while len(self.lines) <= self.start and self.proc.poll() is None and time.time() - t0 < 1:
                time.sleep(0.002)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[self.start:]:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(ns, precision):
    """Bytes per point per RK stage (each array element once per stage):
    n_var*(Q^k + Q^n + Q^(k+1)) + 2*T + 10*geometry, at the stored widths."""
    nv = 5 + ns
    if precision == "fp64":
        return nv * 24 + 2 * 8 + 10 * 8
    return nv * 24 + 2 * 4 + 10 * 4


def field_errors(b, b0):
    """Relative L2 / Linf errors of the primitives b against b0 ([6][n]):
    rho, p, T against themselves, the velocity components against the
    velocity magnitude (a component that starts at zero has no scale of its
    own)."""
    out = {}
    vmag = np.sqrt(b0[1] ** 2 + b0[2] ** 2 + b0[3] ** 2)
    for i, nm in enumerate(["rho", "u", "v", "w", "p", "T"]):
        ref = vmag if 1 <= i <= 3 else b0[i]
        out["l2_" + nm] = float(np.linalg.norm(b[i] - b0[i]) / np.linalg.norm(ref))
        out["linf_" + nm] = float(np.abs(b[i] - b0[i]).max() / np.abs(ref).max())
    return out


def face_kernel_bytes(ns, precision, dq=False):
    """Bytes per point of the face kernel: it reads the primitives (6+ns),
    transport (2+ns) and geometry (10) once and writes three faces of n_var
    fluxes (split variants) or the point's residual of n_var values (the dq
    variant, which differences the faces inside its tile), at the bulk width."""
    w = 8 if precision == "fp64" else 4
    return ((6 + ns) + (2 + ns) + 10 + (1 if dq else 3) * (5 + ns)) * w


def ncu_traffic(kernel_tag):
    """DRAM bytes per stage-kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "%s.txt" % kernel_tag)
    try:
        for ln in open(path):
            if ln.startswith("dram_bytes_per_launch:"):
                return float(ln.split(":")[1])
    except Exception:
        pass
    return None


def ncu_instructions_per_point():
    """Thread instructions per point of the TMA face kernel (FP32, 9 species)
    from the committed ncu instruction-mix summary."""
    path = os.path.join(ROOT, "profiles", "faces_update_instruction_mix_box96_mixed.txt")
    try:
        for ln in open(path):
            if ln.startswith("thread_instructions_per_point:"):
                return float(ln.split(":")[1])
    except Exception:
        pass
    return None


def issue_roofline(instr_per_point, npts, kernel_ms, sm_mhz):
    """The face kernel against its instruction-issue bound: every SM issues
    at most 4 warp instructions (128 thread instructions) per cycle."""
    if not instr_per_point or not sm_mhz:
        return None
    import torch
    n_sm = torch.cuda.get_device_properties(0).multi_processor_count
    peak = n_sm * 4 * 32 * sm_mhz * 1e6  # thread instructions per second
    bound_ms = instr_per_point * npts / peak * 1e3
    return {"thread_instructions_per_point": instr_per_point, "source": "ncu instruction mix (96^3 capture)",
            "issue_bound_ms": bound_ms, "kernel_ms": kernel_ms, "frac": bound_ms / kernel_ms,
            "peak": "%d SMs x 4 schedulers x 32 lanes x %.0f MHz" % (n_sm, sm_mhz)}


def max_over_ranks(ms, dist):
    """The slowest rank's time (replicas run independently; the job takes
    as long as its slowest GPU)."""
    if not dist:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, npts, steps, ms_total):
    """Mcell-updates/s of the whole job: every rank updates npts points 3
    times per step, in the slowest rank's time."""
    return world * npts * 3 * steps / (ms_total / 1e3) / 1e6


def run_ours(args, rank, world, dist):
    import torch
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases

    torch.cuda.set_device(rank % max(1, torch.cuda.device_count()))
    sp = cases.synthetic_species()
    case = cases.case_box(args.n, species=sp, seed=1234)
    out = {}
    states = {}
    for prec in ("fp64", "mixed"):
        d = cc.Driver.from_case(case, prec)
        if args.variant != "auto":  # the fused TMA and dq variants exist in the FP32 bulk precision only
            fp32_only = args.variant in ("tma", "dq-tma")
            d.set_tuning("split-tma-p" if prec == "fp64" and fp32_only else args.variant, args.kz, args.tile_j)
        d.initialize_computation()
        s = torch.cuda.ExternalStream(d.stream())
        info = d.info()
        npts = info["n_points"]
        d.simulate(args.warmup)
        d.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(s)
            d.simulate(args.steps)
            e1.record(s)
            e1.synchronize()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist)
        kt = d.time_kernels(2)
        out[prec] = {"ms_total": ms, "ms_per_step": ms / args.steps, "npts": npts, "clocks": clk.summary(),
                     "kernels": kt, "info": info, "status": d.status(), "tuning": d.tuning()}
        d.close()
    # mixed vs FP64 error after err_steps steps from the same state
    errs = {}
    if args.err_steps > 0 and rank == 0:
        res = {}
        for prec in ("fp64", "mixed"):
            d = cc.Driver.from_case(case, prec)
            d.set_renormalize(True)  # same algorithm in both precisions
            d.initialize_computation()
            d.simulate(args.err_steps)
            bv, yk, cv = d.field[0].get_state()
            res[prec] = (bv, yk)
            d.close()
        n = args.n
        sl = lambda a: a.reshape(a.shape[0], n + 4, n + 4, n + 4)[:, 2:-2, 2:-2, 2:-2].reshape(a.shape[0], -1)
        b64, b32 = sl(res["fp64"][0]), sl(res["mixed"][0])
        y64, y32 = sl(res["fp64"][1]), sl(res["mixed"][1])
        l2 = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        li = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
        errs = {"steps": args.err_steps, "reference": "FP64 run of the same scheme (Y renormalised in FP64)",
                "velocity_norm": "u, v, w errors relative to the velocity magnitude |V| of the FP64 run"}
        errs.update(field_errors(b32, b64))
        errs["l2_Y"] = l2(y32, y64)
        errs["linf_Y"] = li(y32, y64)
        for k, nm in enumerate(sp["names"]):
            errs["l2_Y_" + nm] = l2(y32[k], y64[k])
            errs["linf_Y_" + nm] = li(y32[k], y64[k])
    # end to end through the C ABI with host buffers (mixed), as a caller of
    # the workload runs it: the initial state uploaded from pinned host memory,
    # the workload's E_STEPS steps, each computing the residual and copying it
    # into pinned host memory without waiting (cc_residual_async), and the
    # final state downloaded.  The job length is the workload's, not --steps.
    e2e = None
    if rank == 0:
        blk = case["blocks"][0]
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
        bv_h, yk_h = pin(blk["bv"]), pin(blk["yk"])
        d = cc.Driver.from_case(case, "mixed")
        if args.variant != "auto":
            d.set_tuning(args.variant, args.kz, args.tile_j)
        d.initialize_computation()
        d.simulate(2)
        d.sync()
        ng = bv_h.shape[1]
        bv_o = pin(np.empty_like(bv_h))
        yk_o = pin(np.empty_like(yk_h))
        cv_o = pin(np.empty((14, ng)))
        K = args.e2e_steps
        res_h = pin(np.zeros((K, 4)))
        t0 = time.perf_counter()
        d.field[0].set_state(bv_h, yk_h)
        for s in range(K):
            d.simulate(1, residual=True)
            cc._check(d.lib.cc_residual_async(d.ctx, res_h[s].ctypes.data_as(cc._dp)))
        cc._check(d.lib.cc_get_state(d.ctx, 0, cc._ptr(bv_o), cc._ptr(yk_o), cc._ptr(cv_o), 0))
        dt = time.perf_counter() - t0
        assert np.isfinite(res_h).all() and (res_h[:, 0] > 0).all()
        npts = out["mixed"]["npts"]
        up = bv_h.nbytes + yk_h.nbytes
        down = bv_o.nbytes + yk_o.nbytes + cv_o.nbytes + res_h.nbytes
        e2e = {"value": npts * 3 * K / dt / 1e6, "unit": "Mcell-updates/s", "h2d_bytes_per_step": up / K,
               "d2h_bytes_per_step": down / K, "steps": K,
               "timing": "host wall clock around the whole job: state upload from pinned memory, %d steps with "
                         "the residual of every step copied to pinned memory asynchronously, state download" % K}
        d.close()
    return out, errs, e2e


def run_multiblock(args):
    """64 uneven blocks (4x4x4 periodic layout, 16..96 points per side): the
    batched launch (one launch per stage kernel over all blocks, one CUDA
    graph per step) against one launch per block per kernel, both precisions."""
    import torch
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases

    case = cases.case_multiblock64(seed=2024, species=cases.synthetic_species())
    res = {}
    for prec in ("mixed", "fp64"):
        for mode in ("batched", "per_block"):
            d = cc.Driver.from_case(case, prec)
            d.set_launch_mode(mode)
            d.initialize_computation()
            s = torch.cuda.ExternalStream(d.stream())
            npts = d.info()["n_points"]
            d.simulate(args.warmup)
            d.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            with ClockSampler(torch.cuda.current_device()) as clk:
                e0.record(s)
                d.simulate(args.steps)
                e1.record(s)
                e1.synchronize()
            ms = e0.elapsed_time(e1)
            res[(prec, mode)] = {"value": npts * 3 * args.steps / (ms / 1e3) / 1e6, "ms_per_step": ms / args.steps,
                                 "npts": npts, "clocks": clk.summary(), "tuning": d.tuning(), "status": d.status()}
            d.close()
    b = res[("mixed", "batched")]
    peaks, peak_kind = load_peaks()
    line = {"metric": METRIC, "value": b["value"], "unit": "Mcell-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": b["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 fluxes/transport + f64 conserved/Newton/reductions",
            "data": "synthetic",
            "config": {"workload": "multiblock64_9sp_viscous_rk3", "blocks": len(case["blocks"]),
                       "block_sizes_per_axis": cases.multiblock_sizes(2024), "points": b["npts"],
                       "precision": "mixed", "parallelism": "single GPU", "l2": "inputs larger than L2 (no flush)",
                       "graph": "one CUDA graph per step"},
            "per_block_launches": {k[0]: {"batched": res[(k[0], "batched")]["value"],
                                          "per_block": res[(k[0], "per_block")]["value"],
                                          "batched_over_per_block": res[(k[0], "batched")]["value"]
                                          / res[(k[0], "per_block")]["value"]} for k in res},
            "plain_fp64": {"value": res[("fp64", "batched")]["value"], "unit": "Mcell-updates/s"},
            "mixed_over_fp64": b["value"] / res[("fp64", "batched")]["value"],
            "clocks": b["clocks"], "autotune": {"mixed": b["tuning"], "fp64": res[("fp64", "batched")]["tuning"]},
            "status": {"%s/%s" % k: v["status"] for k, v in res.items()}}
    print(json.dumps(line), flush=True)


def run_lusgs(args):
    """LU-SGS steady steps (the implicit scheme of temporal_scheme 1) on the
    128^3 box at CFL 5, both precisions: step time from CUDA events around
    graph replays, and the split of a step from an event-timed run (face
    kernels; right-hand side + 2 x (mx+my+mz-2) sweep hyperplanes + update;
    halo program)."""
    import torch
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases

    case = cases.case_box(args.n, species=cases.synthetic_species(), seed=1234)
    case["params"]["cfl"] = 5.0
    res = {}
    for prec in ("mixed", "fp64"):
        d = cc.Driver.from_case(case, prec)
        d.initialize_computation()
        s = torch.cuda.ExternalStream(d.stream())
        npts = d.info()["n_points"]
        d.simulate(args.warmup, "lusgs")
        d.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(s)
            d.simulate(args.steps, "lusgs")
            e1.record(s)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        kt = d.time_kernels(2, "lusgs")
        res[prec] = {"value": npts * args.steps / (ms / 1e3) / 1e6, "ms_per_step": ms / args.steps,
                     "split_ms": {"faces": kt["faces_ms"], "rhs_sweeps_update": kt["update_ms"],
                                  "halo": kt["halo_ms"]},
                     "clocks": clk.summary(), "status": d.status(), "npts": npts}
        d.close()
    m = res["mixed"]
    n = args.n
    line = {"metric": "Mcell-updates/s per LU-SGS steady step", "value": m["value"], "unit": "Mcell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fluxes/transport + f64 conserved/sweeps/Newton", "data": "synthetic",
            "config": {"workload": "box%d_9sp_viscous_lusgs" % n, "grid": "%d^3 points, 2 mm periodic cube" % n,
                       "scheme": "LU-SGS, local time step, CFL 5", "precision": "mixed",
                       "sweep_launches_per_step": 2 * (3 * n - 2), "l2": "inputs larger than L2 (no flush)",
                       "graph": "one CUDA graph per step"},
            "split_ms": m["split_ms"], "plain_fp64": {k: res["fp64"][k] for k in ("value", "ms_per_step", "split_ms")},
            "clocks": m["clocks"], "status": {k: v["status"] for k, v in res.items()}}
    print(json.dumps(line), flush=True)


def run_mixing_layer(args):
    """Precision study on the 1024x512x4 H2/air temporal mixing layer: FP64,
    mixed and full-FP32 runs from the same state (Y renormalised in all
    three), relative L2 / Linf errors of the primitives against FP64 at the
    snapshot steps, and each precision's throughput over the last segment."""
    import torch
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases

    case = cases.case_mixing_layer(1024, 512, 4, species=cases.synthetic_species())
    snaps = [int(x) for x in args.study_steps.split(",")]
    nx, ny, nz = case["blocks"][0]["dims"]
    sl = lambda a: a.reshape(a.shape[0], nz + 4, ny + 4, nx + 4)[:, 2:-2, 2:-2, 2:-2].reshape(a.shape[0], -1)
    states, perf, status = {}, {}, {}
    for prec in ("fp64", "mixed", "fp32"):
        d = cc.Driver.from_case(case, prec)
        d.set_renormalize(True)
        d.initialize_computation()
        s = torch.cuda.ExternalStream(d.stream())
        npts = d.info()["n_points"]
        done, states[prec] = 0, {}
        for k in snaps:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            d.simulate(k - done)
            e1.record(s)
            e1.synchronize()
            perf[prec] = {"value": npts * 3 * (k - done) / (e0.elapsed_time(e1) / 1e3) / 1e6,
                          "steps_timed": "%d-%d" % (done, k)}
            done = k
            bv, yk, _ = d.field[0].get_state()
            states[prec][k] = (sl(bv), sl(yk))
        status[prec] = d.status()
        d.close()
    l2 = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    li = lambda a, b: float(np.abs(a - b).max() / np.abs(b).max())
    errors = {}
    for prec in ("mixed", "fp32"):
        errors[prec] = {}
        for k in snaps:
            (b, y), (b0, y0) = states[prec][k], states["fp64"][k]
            e = field_errors(b, b0)
            e["l2_Y"], e["linf_Y"] = l2(y, y0), li(y, y0)
            errors[prec][str(k)] = e
    m = perf["mixed"]
    line = {"metric": METRIC, "value": m["value"], "unit": "Mcell-updates/s", "n_gpus": 1, "steps": snaps[-1],
            "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 fluxes/transport + f64 conserved/Newton/reductions", "data": "synthetic",
            "config": {"workload": "mixing_layer_1024x512x4_9sp_viscous_rk3", "streams": case["streams"],
                       "bc": "periodic x and z, zero-gradient outflow in y", "precision": "mixed",
                       "l2": "inputs larger than L2 (no flush)", "graph": "one CUDA graph per step"},
            "throughput": perf, "mixed_over_fp64": m["value"] / perf["fp64"]["value"],
            "errors_vs_fp64": errors, "status": status}
    print(json.dumps(line), flush=True)


def run_closure(args):
    """256^3 box (the 128^3 workload's generator), mixed precision: stages
    with the exact Wilke / constant-Schmidt transport against stages with the
    learned closure on the tensor cores (exact fallback outside its hull);
    throughput, fallback rate, closure accuracy on fresh states and the
    difference of the two solutions."""
    import torch
    import combustioncodegpu_b200 as cc
    from combustioncodegpu_b200 import cases, closure

    sp = cases.synthetic_species()
    n = 256
    case = cases.case_box(n, species=sp, seed=1234)
    w, report = closure.load()
    res, states = {}, {}
    for mode in ("exact", "closure"):
        d = cc.Driver.from_case(case, "mixed")
        if mode == "closure":
            d.set_closure(w)
            d.use_closure(True)
        d.initialize_computation()
        s = torch.cuda.ExternalStream(d.stream())
        npts = d.info()["n_points"]
        d.simulate(args.warmup)
        d.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(s)
            d.simulate(args.steps)
            e1.record(s)
            e1.synchronize()
        ms = e0.elapsed_time(e1)
        kt = d.time_kernels(1)
        res[mode] = {"value": npts * 3 * args.steps / (ms / 1e3) / 1e6, "ms_per_step": ms / args.steps,
                     "kernels": kt, "clocks": clk.summary(), "status": d.status(), "tuning": d.tuning()}
        if mode == "closure":
            n_eval, n_fb, n_chk = d.closure_stats()
            res[mode]["closure_points"] = n_eval
            res[mode]["fallback_rate"] = (n_fb + n_chk) / max(1, n_eval)
            res[mode]["fallback_rate_outside_hull"] = n_fb / max(1, n_eval)
            res[mode]["fallback_rate_run_time_check"] = n_chk / max(1, n_eval)
            res[mode]["run_time_check"] = "4 samples per 128-point tile against the exact transport, bound 1e-3"
            d.set_closure_bound(0.0)  # the network alone
            res[mode]["closure_accuracy_fresh_states"] = closure.validate(d, sp, n=200_000, seed=31)
            res[mode]["closure_accuracy_box_states"] = closure.validate(d, sp, n=200_000, seed=31, states="box")
        states[mode] = d.field[0].get_state()[0]
        d.close()
    sl = lambda a: a.reshape(6, n + 4, n + 4, n + 4)[:, 2:-2, 2:-2, 2:-2].reshape(6, -1)
    diff = field_errors(sl(states["closure"]), sl(states["exact"]))
    c = res["closure"]
    line = {"metric": METRIC, "value": c["value"], "unit": "Mcell-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": c["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 fluxes + bf16 tensor-core transport closure + f64 conserved/Newton",
            "data": "synthetic",
            "config": {"workload": "box256_9sp_viscous_rk3_closure", "grid": "256^3 points, 2 mm periodic cube",
                       "closure": "MLP (T, X_1..9) -> (mu, lambda, rhoD_1..9), 3x64 SiLU, BF16 weights, "
                                  "BF16 hi/lo activations, tcgen05 FP32 accumulate", "precision": "mixed",
                       "l2": "inputs larger than L2 (no flush)", "graph": "one CUDA graph per step"},
            "exact_transport": res["exact"], "closure": c,
            "closure_over_exact": c["value"] / res["exact"]["value"],
            "solution_difference_after_steps": diff,
            "training": {k: report[k] for k in ("n_samples", "epochs", "seconds_train", "torch_model_rel_err")}}
    print(json.dumps(line), flush=True)


def reference_kernels_b200(n, steps):
    """The reference's own CUDA kernels, FP64, timed on this GPU: built from
    the reference sources into oracle/_ref/ref_harness_ms by
    oracle/ref_harness/build_ref.sh (with the three patches of its header) and
    driven by its harness on the n^3 box of the workload's generator.  The
    harness times `steps` explicit steps after one warm-up step with CUDA
    events: the per-block kernels of a step alone (the reference's one
    launch per block per kernel: set_dq_to_0, inviscid and viscous fluxes,
    local time step, update_cv_and_bv, update_physical_properties), and with
    the boundary launches and the harness's interface fill.  One explicit step
    is one stage of work, so Mcell-updates/s per stage = points / step time."""
    import tempfile
    from combustioncodegpu_b200 import cases
    from oracle.ref_harness.case_file import write_case

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness_ms")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_harness_ms is not built (it needs the reference sources)"}
    case = cases.case_box(n, species=cases.synthetic_species(), seed=1234)
    case["n_steps"] = 1
    with tempfile.TemporaryDirectory() as d:
        cf, of = os.path.join(d, "case.bin"), os.path.join(d, "out.bin")
        write_case(cf, case)
        r = subprocess.run([exe, cf, of, "--time", str(steps)], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"unavailable": "harness exit %d: %s" % (r.returncode, (r.stderr or r.stdout).strip()[-200:])}
    t = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    pts = t["points"]
    return {"grid": "%d^3 points, same generator and seed as the workload" % n, "precision": "fp64",
            "steps_timed": steps, "kernels_ms_per_step": t["kernels_ms_per_step"],
            "step_ms_with_halo_fill": t["step_ms_with_halo_fill"],
            "value": pts / (t["kernels_ms_per_step"] / 1e3) / 1e6, "unit": "Mcell-updates/s per stage",
            "timing": "CUDA events around the reference's per-block kernel launches (one explicit step = one "
                      "stage of work)"}


def cpu_baseline(args, n_threads, steps=1, n=64):
    """The oracle on the host cores: bounded sample of the workload (an
    n^3-point box with the same per-point work, `steps` RK3 steps)."""
    from combustioncodegpu_b200 import cases
    from oracle.oracle_py import Oracle

    case = cases.case_box(n, species=cases.synthetic_species(), seed=1234)
    o = Oracle(case, threads=n_threads)
    o.init()
    t0 = time.perf_counter()
    o.rk3_step(steps)
    dt = time.perf_counter() - t0
    pts = n ** 3
    return {"value": pts * 3 * steps / dt / 1e6, "unit": "Mcell-updates/s", "cores": n_threads, "kind": "port",
            "sample": "%d^3-point box, same 9-species viscous workload, %d RK3 step(s), FP64" % (n, steps),
            "seconds": dt}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as tdist
        import datetime
        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    n_threads = os.cpu_count() or 1
    if args.impl == "reference":
        if rank == 0:
            per_step = []
            for _ in range(args.warmup):
                cpu_baseline(args, n_threads)
            for _ in range(max(1, args.steps)):
                per_step.append(cpu_baseline(args, n_threads))
            v = float(np.median([r["value"] for r in per_step]))
            base = per_step[0]
            line = {"metric": METRIC, "value": v, "unit": "Mcell-updates/s", "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": float(np.median([r["seconds"] for r in per_step])) * 1e3,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "impl": "reference",
                    "config": {"workload": WORKLOAD, "grid": "%d^3 points sampled as 64^3" % args.n, "species": 9},
                    "cpu_baseline": {"value": v, "unit": "Mcell-updates/s", "cores": n_threads, "kind": "port",
                                     "sample": base["sample"]},
                    "e2e": {"value": v, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    if args.workload in ("multiblock64", "mixing_layer", "box256_closure", "box128_lusgs"):
        if rank == 0:
            {"multiblock64": run_multiblock, "mixing_layer": run_mixing_layer,
             "box256_closure": run_closure, "box128_lusgs": run_lusgs}[args.workload](args)
        if dist:
            dist.destroy_process_group()
        return
    out, errs, e2e = run_ours(args, rank, world, dist)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    peaks, peak_kind = load_peaks()
    mixed, plain = out["mixed"], out["fp64"]
    value = whole_job_rate(world, mixed["npts"], args.steps, mixed["ms_total"])
    value_plain = whole_job_rate(world, plain["npts"], args.steps, plain["ms_total"])
    bpp = algorithmic_bytes(9, "mixed")
    kt = mixed["kernels"]
    stage_ms = kt["stage_ms"]
    variant = mixed["tuning"]["variant"]
    split = variant in ("split", "split-tma", "split-tma-p", "dq-tma")
    stage_achieved = bpp * mixed["npts"] / (stage_ms / 1e3) / 1e9
    if variant == "dq-tma":  # dominant kernel: the face kernel that writes dq
        ty = mixed["tuning"]["tile"][1]
        kname = "k_faces_dq<float,9,%d,%d>" % (ty, {4: 2, 8: 3, 16: 1}[ty])
        kbpp, kms = face_kernel_bytes(9, "mixed", dq=True), kt["faces_ms"]
        traffic = ncu_traffic("faces_dq_kernel_box128_mixed")
    elif split:  # dominant kernel: the face kernel
        tma = variant in ("split-tma", "split-tma-p")
        kname = "k_faces_tma<float,9>" if tma else "k_faces<float,9>"
        kbpp, kms = face_kernel_bytes(9, "mixed"), kt["faces_ms"]
        traffic = ncu_traffic("faces_tma_kernel_box128_mixed" if tma else "faces_kernel_box128_mixed")
    else:
        kname, kbpp, kms = "k_stage<float,9>", bpp, stage_ms
        traffic = ncu_traffic("stage_kernel_box128_mixed")
    achieved = kbpp * mixed["npts"] / (kms / 1e3) / 1e9
    cpu = cpu_baseline(args, os.cpu_count() or 1, steps=2, n=96)
    refk = reference_kernels_b200(args.ref_n, args.ref_steps) if args.ref_n > 0 else None
    if refk and "value" in refk:
        refk["ours_mixed_over_reference"] = value / refk["value"]
        refk["ours_fp64_over_reference"] = value_plain / refk["value"]
    levels = mixed["info"]["halo_levels"]
    # per stage: the stage kernels and the halo program (the node levels in
    # one cooperative launch, or one per level beyond 8 levels, then one launch
    # of the copies with the post-exchange time step); per step: the
    # time-step finalisation
    n_stage = {"l1": 1, "tma": 1, "split": 2, "split-tma": 3, "split-tma-p": 3, "dq-tma": 2}[variant]
    halo = (min(levels, 1) if levels <= 8 else levels) + 1
    launches_per_step = 3 * (n_stage + halo) + 1
    line = {
        "metric": METRIC, "value": value, "unit": "Mcell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mixed["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 fluxes/transport + f64 conserved/Newton/reductions", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": "%d^3 points, 2 mm periodic cube" % args.n, "species": 9,
                   "unique_points": "%d^3: the vertex-centred periodic box shares its end layer on each axis" %
                                    (args.n - 1),
                   "scheme": "MUSCL-minmod + AUSM+ + 2nd-order viscous, SSP-RK3, CFL 0.5",
                   "precision": "mixed", "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (no flush)", "graph": "one CUDA graph per step"},
        "plain_fp64": {"value": value_plain, "unit": "Mcell-updates/s", "ms_per_step": plain["ms_per_step"]},
        "mixed_over_fp64": value / value_plain,
        "error_mixed_vs_fp64": errs,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "kernel": kname, "algorithmic_bytes_per_point": kbpp, "kernel_ms_per_launch": kms,
                     "peak_kind": peak_kind,
                     "issue": (issue_roofline(ncu_instructions_per_point(), mixed["npts"], kms,
                                              mixed["clocks"].get("sm_mhz")) if kname.startswith("k_faces_tma")
                               else None),
                     "stage": {"ms": stage_ms, "faces_ms": kt["faces_ms"], "update_ms": kt["update_ms"],
                               "algorithmic_bytes_per_point": bpp, "achieved_gbs": stage_achieved,
                               "frac": stage_achieved / peaks["hbm_gbs"]}},
        "cpu_baseline": {"value": cpu["value"], "unit": cpu["unit"], "cores": cpu["cores"], "kind": cpu["kind"],
                         "sample": cpu["sample"]},
        "e2e": e2e,
        "reference_kernels_b200": refk,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": mixed["clocks"],
        "status": {"mixed": mixed["status"], "fp64": plain["status"]},
        "autotune": {"mixed": mixed["tuning"], "fp64": plain["tuning"]},
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
