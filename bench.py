#!/usr/bin/env python3
"""Benchmark: CNAB2 steps/s of the full MHD shell step at lmax=255, nr=129
(nlat=384, nlon=768; fields u_tor, u_pol, B_tor, B_pol, T), graph-captured on
one B200 per rank.

One "step" is step_once! (scripts/bench_timestepping.jl:6-18): temperature,
velocity and magnetic nonlinear terms (4 scalar + 4 vector syntheses, 1 scalar
+ 2 vector analyses, the grid products) and the five CNAB2 banded solves.

Arms:
  default            this package through its C ABI (libgdb200.so)
  --impl reference   the FP64 CPU restatement of the reference step (oracle/),
                     timed on the host cores at the full headline size
                     (lmax 255, nr 129): 1 warm-up and up to 5 timed steps on
                     all cores, and 1 timed step on one thread.

Other measurements (one JSON line each, instead of the headline):
  --transforms       the transform-only batch (lmax 127, 97 shells x 9 fields):
                     errors against the oracle and device times, FP64 and mixed
  --adjoint          the adjoint configuration's gradient against FP64 finite
                     differences and the oracle's forward mode, with timings
  --ensemble N       the batched uneven ensemble of N shells
  --scheme S         the headline step under ts_scheme = S (cnab2, eab2, erk2)
  --workload W       a smaller named shell for profiling captures

Multi-GPU (torchrun): by default every rank runs an independent replica of the
same workload (weak scaling; value = N x steps / max-over-ranks time).
  --decomposed       one model across the ranks (strong scaling): each rank
                     owns whole m columns for the radial derivatives and CNAB2
                     and a slab of shells for the transforms and products, with
                     two NCCL all-to-alls per step through device buffers
                     (distributed.DistributedStep); time = max over ranks
"""
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
sys.path.insert(0, os.path.join(ROOT, "geodynamo.jl_b200"))

METRIC = "CNAB2 steps/s lmax255 nr129: mixed-prec vs FP64 GPU at 1e-9 energy err"
WORKLOAD = "shell_l255_nr129"


def load_package():
    import importlib.util
    if "gdb200" in sys.modules:
        return sys.modules["gdb200"]
    pkg_dir = os.path.join(ROOT, "geodynamo.jl_b200")
    spec = importlib.util.spec_from_file_location("gdb200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gdb200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload_params():
    import workloads
    c = dict(workloads.CONFIGS[WORKLOAD])
    c.update(workloads.SHELL_PHYSICS)
    return c


# ---------------------------------------------------------------------------
# algorithmic work per kernel launch (bytes or flops), for the roofline
# ---------------------------------------------------------------------------
def kernel_work(name, p, nlm, precision):
    """Algorithmic work of one launch: {"flops": F or None, "bytes": B or None}.

    Legendre: flops count the contraction once (not the three split-TF32
    products); bytes are the coefficients, the Fourier components and the
    table (images) each read or written once."""
    L, nlat, nlon, nr = p["lmax"], p["nlat"], p["nlon"], p["nr"]
    if name.endswith("_fp64"):
        precision = "fp64"                    # an FP64 stage (also inside the mixed step)
    nth = nlat // 2
    G = nlat * nlon * nr                      # grid points per field
    F = nr * (L + 1) * nlat                   # Fourier coefficients per component
    S = 2 * nr * nlm                          # spectral doubles per field
    rb = 8 if precision == "fp64" else 4      # grid real bytes
    cb = 2 * rb                               # Fourier complex bytes
    if precision == "fp64":
        table = nlm * nth * 8                 # one FP64 table [mode][north colatitude]
        synth_table = anal_table = table
    else:
        chunk = 32768                         # split-TF32 hi + lo image chunk of 128 x 32
        ntile = -(-nth // 128)
        nck = lambda k: -(-k // 32)  # noqa: E731
        synth_table = chunk * ntile * sum(nck((L - m + 2) // 2) + nck((L - m + 1) // 2) for m in range(L + 1))
        anal_table = chunk * (L + 1) * 2 * (-(-nth // 32))
    legendre = {
        "legendre_synth_scalar": (2.0 * nlm * nlat * nr * 4, 4 * S * 8 + 4 * F * cb + synth_table),
        "legendre_synth_vector": (8.0 * nlm * nlat * nr, 2 * S * 8 + 2 * F * cb + 2 * synth_table),
        "legendre_analysis_scalar": (2.0 * nlm * nlat * nr, F * cb + S * 8 + anal_table),
        "legendre_analysis_vector": (8.0 * nlm * nlat * nr, 2 * F * cb + 2 * S * 8 + 2 * anal_table),
    }
    if name == "legendre_synth_vector_i8":
        # int8 digit slices (6 digits): 21 int8 products per FP64 product; bytes:
        # the FP64 coefficients, the FP64 Fourier output and its FP32 copy, the
        # coefficient digit images (written, then read once per colatitude
        # tile) and the table digit images
        ksteps = sum(-(-((L - m + 2) // 2) // 32) + -(-((L - m + 1) // 2) // 32) for m in range(L + 1))
        ncb = -(-4 * nr // 32)
        b_img = ksteps * ncb * 6 * 32 * 32
        a_img = ksteps * (-(-nth // 64)) * 6 * 128 * 32
        return {"flops": 8.0 * nlm * nlat * nr * 21, "int8": True,
                "bytes": 2 * S * 8 + 2 * F * 16 + 2 * F * 8 + b_img * (1 + -(-nth // 64)) + a_img}
    for k, (fl, by) in legendre.items():
        if name.startswith(k):
            return {"flops": fl, "bytes": by}
    table = {
        # fused phase kernels: blocked Fourier components in, folded transforms out
        "fused_temperature": 5 * F * cb + F * cb,
        "fused_velocity": 8 * F * cb + 2 * F * cb,
        "fused_induction": 4 * F * cb + 2 * F * cb,
        "nl_temperature": 6 * G * rb,
        "nl_velocity": 10 * G * rb,
        "nl_induction": 6 * G * rb,
        "nl_coriolis": 4 * G * rb,
        # FP64 <-> blocked FP32 Fourier components (2) and the folded-transform widening (2)
        "fourier_convert": 2 * F * (16 + 8),
        "fold_convert": 2 * F * (8 + 16 + 16),
        # per field: read u, N, N_prev, write u (the history roll is a bank switch)
        "cnab2_solve": 5 * 4 * S * 8,
        # the same arrays plus the exponential cache (3 kinds x (L+1) x [E | phi1])
        "eab2_update": 5 * 4 * S * 8 + 3 * (L + 1) * 2 * nr * nr * 8,
        # linear = E u, k1 = phi1 N, stage = E_h u + phi1_h N over u: 7 arrays per field, 4 matrices
        "erk2_prepare": 5 * 7 * S * 8 + 3 * (L + 1) * 4 * nr * nr * 8,
        # u = linear + dt (k1 + phi2 (N_stage - N)): 5 arrays per field, 1 matrix
        "erk2_finalize": 5 * 5 * S * 8 + 3 * (L + 1) * nr * nr * 8,
        "spectral_gradients": 4 * S * 8,
        "spectral_curl": 4 * S * 8,
        "temperature_bc": 4 * nlm * 8,
    }
    for k, v in table.items():
        if name.startswith(k):
            # per field and (l, m, plane) column: EAB2 one n x 2n matrix-vector
            # product, the ERK2 prepare four n x n ones, the finalize one
            mv = {"eab2_update": 2, "erk2_prepare": 4, "erk2_finalize": 1}.get(k)
            flops = 5 * S * 2.0 * mv * nr if mv else None
            return {"flops": flops, "bytes": v}
    return None


def fp64_gemm_tflops(n=4096, reps=5):
    """cuBLAS FP64 GEMM rate (torch.matmul, n^3, best of reps, CUDA events):
    the measured peak the FP64 step's tensor-core contractions are rated against."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def measured_traffic(name):
    """DRAM bytes per launch of a kernel from the committed ncu summary of the
    headline workload (profiles/dram_traffic_shell_l255_nr129.txt), or None."""
    if WORKLOAD != "shell_l255_nr129":
        return None
    try:
        for line in open(os.path.join(ROOT, "profiles", "dram_traffic_shell_l255_nr129.txt")):
            f = line.split()
            if len(f) >= 2 and not line.startswith("#") and f[0] == name:
                return float(f[1])
    except OSError:
        pass
    return None


def fft_bytes(p, ncomp, precision):
    L, nlat, nlon, nr = p["lmax"], p["nlat"], p["nlon"], p["nr"]
    rb = 8 if precision == "fp64" else 4
    return ncomp * (nr * (L + 1) * nlat * 2 * rb + nr * nlat * nlon * rb)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_reference_rate(steps, warmup, threads=None):
    """Oracle steps/s on the workload's full grid (every shell), timed on the
    host cores: `warmup` untimed steps, then `steps` timed ones; threads None =
    all cores.  Returns (steps/s, seconds per step, threads used)."""
    from oracle.oracle import Oracle
    import workloads
    p = workload_params()
    nr = p["nr"]
    o = Oracle(lmax=p["lmax"], nlat=p["nlat"], nlon=p["nlon"], nr=nr, dt=p["dt"], threads=threads)
    for k, (a, b) in workloads.seeded_state(p["lmax"], p["lmax"], nr, seed=0).items():
        o.set_field(k, a, b)
    for _ in range(warmup):
        o.step(1)
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(1)
    dt = (time.perf_counter() - t0) / steps
    del o
    return 1.0 / dt, dt, os.cpu_count() if threads is None else threads


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # the full headline size (about 5 s per step on 16 host cores, about a
    # minute on one): 1 warm-up and at most 5 timed steps on all cores, then 1
    # timed step on one thread
    p = workload_params()
    steps = max(1, min(args.steps, 5))
    warm = 1
    rate, dt_all, cores = cpu_reference_rate(steps, warm)
    rate1, dt_one, _ = cpu_reference_rate(1, 0, threads=1)
    sample = (f"oracle (C++ FP64 restatement of step_once!) at the full {WORKLOAD} grid (lmax={p['lmax']} "
              f"nlat={p['nlat']} nlon={p['nlon']} nr={p['nr']}): {steps} timed steps after {warm} warm-up on "
              f"{cores} threads ({dt_all:.2f} s per step); 1 thread: 1 timed step ({dt_one:.1f} s)")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 / rate, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, default_rng(0))",
            "config": {"workload": WORKLOAD, "lmax": p["lmax"], "nlat": p["nlat"], "nlon": p["nlon"], "nr": p["nr"]},
            "cpu_baseline": {"value": rate, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sample,
                             "one_thread": {"value": rate1, "unit": "steps/s", "cores": 1}},
            "e2e": {"value": rate, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ensemble(args, gdb, workloads, torch, world=1, rank=0):
    """Batched uneven ensemble: args.ensemble seeded shells (lmax 31-95, nr 33-65,
    E and Ra drawn per member), one graph launch per step for all of them;
    aggregate instance-steps/s, device-timed with CUDA events on the ensemble's
    stream, FP64 and mixed precision.  Over several ranks (torchrun) the whole
    instances are dealt round-robin to the ranks (no collective in the step);
    time = max over ranks, value = all instances' steps / that time.
    Members of one lmax share a segmented handle (up to --ensemble-group per
    handle, each with its own radial grid, operators and Coriolis factor); the
    per-member-handle ensemble is timed beside it."""
    allc = workloads.ensemble_draw(args.ensemble)
    mine = list(range(rank, len(allc), world))
    cfgs = [allc[i] for i in mine]
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = {}
    group = max(1, args.ensemble_group)
    legs = [("fp64", group), ("mixed", group)]
    if group > 1:
        legs += [("fp64", 1), ("mixed", 1)]
    for prec, grp in legs:
        ens = gdb.Ensemble(cfgs, precision=prec, group=grp)
        for i, c, m in zip(mine, cfgs, ens.members):
            for k, (a, b) in workloads.seeded_state(c["lmax"], c["lmax"], c["nr"], seed=i).items():
                m.set_field(k, a, b)
        tune = None
        if prec == "mixed":
            # launch shapes chosen by measurement on a scratch copy (members unchanged)
            tms, caps = ens.autotune(5)
            tune = {"ms_per_step": tms, "caps": sorted(set(caps))}
        ens.step(args.warmup)
        if dist is not None:
            dist.barrier()
        ext = torch.cuda.ExternalStream(ens.stream_ptr())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(ext)
        ens.step_async(args.steps)
        e1.record(ext)
        ens.step(0)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ek = sum(m.energy()[0] for m in ens.members)
        if dist is not None:
            t = torch.tensor([ms, ek], dtype=torch.float64, device="cuda")
            dist.all_reduce(t[:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
            ms, ek = float(t[0]), float(t[1])
        key = prec if grp == group else prec + "_handle_per_member"
        res[key] = {"instance_steps_per_s": args.steps * len(allc) / (ms * 1e-3), "ms_per_step": ms / args.steps,
                    "sum_ekin": ek, "handles": len(ens.handles)}
        if tune is not None:
            res[key]["autotune"] = tune
        ens.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": f"ensemble instance-steps/s ({len(allc)} uneven shells)", "value": res["mixed"]["instance_steps_per_s"],
            "unit": "instance-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "scaling": "strong" if world > 1 else "weak",
            "higher_is_better": True, "dtype": "f32/tf32x3 (FP64 solves)", "data": "synthetic (ensemble_draw(seed=3), seeded_state(seed=i))",
            "config": {"workload": "ensemble", "members": len(allc), "lmax": sorted({c["lmax"] for c in allc}),
                       "nr": sorted({c["nr"] for c in allc}), "dt": 1e-5, "ranks": world,
                       "placement": "whole instances round-robin over the ranks",
                       "launch": "one CUDA graph per step; mixed: tensor-core grid caps by gd_ensemble_autotune",
                       "grouping": f"members of one lmax share a segmented handle, <= {group} per handle"},
            **res,
            "ratio_vs_fp64_gpu": res["mixed"]["instance_steps_per_s"] / res["fp64"]["instance_steps_per_s"]}
    print(json.dumps(line), flush=True)
    return 0


def run_decomposed(args, gdb, workloads, torch, world, rank, local):
    """One model stepped across `world` ranks by distributed.DistributedStep over
    NCCL (device exchange buffers); steps/s of that model, time = max over ranks."""
    import datetime
    import torch.distributed as dist
    import distributed as D
    for k, v in (("MASTER_ADDR", "127.0.0.1"), ("MASTER_PORT", "29533"), ("RANK", "0"), ("WORLD_SIZE", "1")):
        os.environ.setdefault(k, v)  # a single rank without torchrun
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device("cuda", local))
    p = workload_params()
    prec = args.precision if args.precision != "auto" else "mixed_vel64"
    keys = ("dt", "rratio", "ekman", "rayleigh", "prandtl", "magnetic_prandtl", "implicit_theta")
    cfg = dict(lmax=p["lmax"], nlat=p["nlat"], nlon=p["nlon"], nr=p["nr"], **{k: p[k] for k in keys})
    ds = D.DistributedStep(gdb, cfg, rank, world, device=local, precision=prec, device_exchange=True)
    for k, (a, b) in workloads.seeded_state(p["lmax"], p["lmax"], p["nr"], seed=0).items():
        ds.set_field(k, a, b)
    ds.step(args.warmup)
    dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    ds.step(args.steps)
    torch.cuda.synchronize()
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t[0]) / args.steps
    ek, em = ds.energy(D.native_l(p["lmax"], p["lmax"]))
    xbytes = ds.dec.exchange_bytes(12) + ds.dec.exchange_bytes(5)
    if rank == 0:
        print(json.dumps({
            "metric": f"CNAB2 steps/s {WORKLOAD} decomposed over {world} ranks", "value": 1e3 / ms,
            "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": prec,
            "data": "synthetic (seeded_state seed 0)",
            "config": {"workload": WORKLOAD, "layout": "m columns (derivatives, CNAB2) / shell slabs (transforms)",
                       "exchange": "NCCL all_to_all_single, device buffers", "exchange_bytes_per_step": xbytes},
            "energy": {"e_kin": ek, "e_mag": em}}), flush=True)
    ds.close()
    dist.destroy_process_group()
    return 0


def run_transforms(args, gdb, workloads, torch):
    """Transform-only configuration: forward + inverse scalar transforms at
    lmax 127 over 97 shells x 9 fields (seeded, (l+1)^-1.5), FP64 and mixed:
    max / RMS relative errors of synthesis, analysis and round trip against
    the FP64 oracle, device time of the transform kernels (per-kernel events)
    and wall time of the host-buffer calls."""
    from oracle.oracle import Oracle
    c = workloads.CONFIGS["transform_l127_nr97x9"]
    L, nlat, nlon, nr, nf = c["lmax"], c["nlat"], c["nlon"], c["nr"], c["nfield"]
    re, im = workloads.transform_batch(L, L, nr, nf, seed=0)
    o = Oracle(lmax=L, nlat=nlat, nlon=nlon, nr=nr)
    grids = np.stack([o.synth_scalar(re[f], im[f]) for f in range(nf)])
    ana = [o.analysis_scalar(grids[f]) for f in range(nf)]
    nlm = re.shape[-1]
    gflop = 2.0 * 2 * nlm * (nlat // 2) * 2 * nr * nf / 1e9  # even/odd-folded Legendre, both directions

    def errs(a, b):
        return (float(np.max(np.abs(a - b)) / np.max(np.abs(b))),
                float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2))))

    res = {}
    for prec in ("fp64", "mixed"):
        g = gdb.SHTnsKitConfig(L, nlat, nlon, nr, precision=prec)
        for _ in range(args.warmup):
            g.analysis_scalar(g.synth_scalar(re, im))
        g.profile_enable(True)
        g.profile_read()
        t0 = time.perf_counter()
        out = g.synth_scalar(re, im)
        back = g.analysis_scalar(grids)
        wall = time.perf_counter() - t0
        prof = g.profile_read()
        g.profile_enable(False)
        rt = g.analysis_scalar(out)
        dev_ms = sum(v[0] for v in prof.values())
        e_s = [errs(out[f], grids[f]) for f in range(nf)]
        e_a = [errs(np.concatenate([back[0][f], back[1][f]]), np.concatenate(ana[f])) for f in range(nf)]
        e_r = [errs(np.concatenate([rt[0][f], rt[1][f]]), np.concatenate([re[f], im[f]])) for f in range(nf)]
        res[prec] = {"synthesis_max": max(e[0] for e in e_s), "synthesis_rms": max(e[1] for e in e_s),
                     "analysis_max": max(e[0] for e in e_a), "analysis_rms": max(e[1] for e in e_a),
                     "roundtrip_max": max(e[0] for e in e_r), "roundtrip_rms": max(e[1] for e in e_r),
                     "device_ms": dev_ms, "wall_ms_host_buffers": wall * 1e3,
                     "legendre_gflops_algorithmic": gflop / (dev_ms * 1e-3),
                     "kernels": {k: v[0] for k, v in prof.items()}}
        g.close()
    line = {"metric": "transform batch forward+inverse (lmax 127, 97 shells x 9 fields)",
            "value": res["mixed"]["device_ms"], "unit": "ms (device, forward+inverse)", "higher_is_better": False,
            "n_gpus": 1, "data": "synthetic (transform_batch(seed=0), (l+1)^-1.5)",
            "config": {"workload": "transform_l127_nr97x9", "lmax": L, "nlat": nlat, "nlon": nlon, "nr": nr,
                       "fields": nf, "legendre_gflop_algorithmic": gflop},
            "fp64": res["fp64"], "mixed": res["mixed"]}
    print(json.dumps(line), flush=True)
    return 0


def run_adjoint(args, gdb, workloads, torch):
    """Adjoint configuration (lmax 63, nr 65, 200 steps, literal boundaries,
    checkpoints every 20 steps): gradient of the r = ro radial-field misfit with
    respect to the initial B_pol, device time of the forward run and of the
    reverse pass, and its agreement with FP64 central finite differences of the
    GPU step on 32 directions and with the forward-mode derivative of the
    oracle's step on 2 of them."""
    c = workloads.CONFIGS["adjoint_l63_nr65"]
    state = workloads.adjoint_state(c["lmax"], c["lmax"], c["nr"], seed=0)

    def make(bpol=None):
        m = gdb.SHTnsKitConfig(c["lmax"], c["nlat"], c["nlon"], c["nr"], dt=c["dt"], bc_mode=c["bc_mode"])
        for k, (a, b) in state.items():
            m.set_field(k, a, b)
        if bpol is not None:
            m.set_field("b_pol", *bpol)
        return m

    m = make()
    tre, tim = workloads.adjoint_target(c["lmax"], c["lmax"], seed=1)
    re = np.zeros(m.spec_shape()); im = np.zeros(m.spec_shape())
    re[-1] = tre; im[-1] = tim
    target = m.synth_scalar(re, im)[-1]
    m.close()
    # timing: forward (200 steps) and the reverse pass on a warm handle
    m = make()
    gdb.magnetic_misfit(m, target, c["steps"], c["checkpoint"])
    for k, (a, b) in state.items():
        m.set_field(k, a, b)
    t0 = time.perf_counter()
    J, gre, gim, ckpt = gdb.magnetic_misfit(m, target, c["steps"], c["checkpoint"])
    t_total = time.perf_counter() - t0
    lam = (np.random.default_rng(0).standard_normal(m.spec_shape()),) * 2
    ext = torch.cuda.ExternalStream(m.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
    m.synchronize(); e0.record(ext)
    m.step_async(c["steps"])
    e1.record(ext); m.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    t1 = time.perf_counter()
    m.magnetic_pullback("b_pol", c["steps"], *lam)
    pull_ms = (time.perf_counter() - t1) * 1e3
    m.close()

    def dot(a, b):
        return float(np.sum(a[0] * b[0]) + np.sum(a[1] * b[1]))

    def misfit(bpol):
        mm = make(bpol)
        mm.step(c["steps"])
        r = gdb.radial_field_outer(mm, *mm.get_field("b_pol")) - target
        mm.close()
        return 0.5 * float(np.sum(r * r))

    b0 = state["b_pol"]
    dirs = workloads.adjoint_directions(c["lmax"], c["lmax"], c["nr"], count=32, seed=2)
    fd_err = []
    for v in dirs:
        eps = 1e-3 * np.sqrt(dot(b0, b0) / dot(v, v))
        fd = (misfit((b0[0] + eps * v[0], b0[1] + eps * v[1])) - misfit((b0[0] - eps * v[0], b0[1] - eps * v[1]))) / (2 * eps)
        ad = dot((gre, gim), v)
        fd_err.append(abs(fd - ad) / abs(ad))
    from oracle.oracle import Oracle
    probe = make()

    def oracle_radial(bpol):
        o = Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], dt=c["dt"], bc_mode=c["bc_mode"])
        for k, (a, b) in state.items():
            o.set_field(k, a, b)
        o.set_field("b_pol", *bpol)
        o.step(c["steps"])
        pre, pim = o.get_field("b_pol")
        f = probe.l_values * (probe.l_values + 1.0) / probe.r[-1] ** 2
        r2 = np.zeros(probe.spec_shape()); i2 = np.zeros(probe.spec_shape())
        r2[-1] = f * pre[-1]; i2[-1] = f * pim[-1]
        return o.synth_scalar(r2, i2)[-1]

    resid = oracle_radial(b0) - target
    fm_err = []
    for v in dirs[:2]:
        fwd = float(np.sum(resid * oracle_radial(v)))
        ad = dot((gre, gim), v)
        fm_err.append(abs(fwd - ad) / abs(ad))
    probe.close()

    # temperature objective: J_T = 1/2 |T(r_mid) - target|^2 after the same 200
    # steps, gradient with respect to the initial temperature by checkpoint and
    # recompute (temperature_misfit), from the seeded temperature of config 0.
    # With the literal operator (bc_mode 0) a nonzero temperature grows by ~1e15
    # in 10 steps at this grid (the configuration's state has none), so this leg
    # uses the Dirichlet rows of bc_mode 2.
    t0s = workloads.seeded_state(c["lmax"], c["lmax"], c["nr"], seed=0)["temp"]
    mid = c["nr"] // 2
    tbc = 2

    def make_t(t0):
        mm = gdb.SHTnsKitConfig(c["lmax"], c["nlat"], c["nlon"], c["nr"], dt=c["dt"], bc_mode=tbc)
        for k, (a, b) in state.items():
            mm.set_field(k, a, b)
        mm.set_field("temp", *t0)
        return mm

    mt = make_t(t0s)
    tgt = np.cos(np.arange(mt.nlon * mt.nlat).reshape(mt.nlon, mt.nlat) * 0.11) * 1e-3
    gdb.temperature_misfit(mt, tgt, c["steps"], c["checkpoint"], shell=mid)  # warm-up (graphs, scratch)
    mt.close()
    mt = make_t(t0s)
    t2 = time.perf_counter()
    JT, tgre, tgim = gdb.temperature_misfit(mt, tgt, c["steps"], c["checkpoint"], shell=mid)
    t_temp = time.perf_counter() - t2
    mt.close()

    def misfit_t(t0):
        mm = make_t(t0)
        mm.step(c["steps"])
        r = mm.synth_scalar(*mm.get_field("temp"))[mid] - tgt
        mm.close()
        return 0.5 * float(np.sum(r * r))

    tdirs = workloads.adjoint_directions(c["lmax"], c["lmax"], c["nr"], count=8, seed=3)
    tfd = []
    for v in tdirs:
        eps = 1e-3 * np.sqrt(dot(t0s, t0s) / dot(v, v))
        fd = (misfit_t((t0s[0] + eps * v[0], t0s[1] + eps * v[1])) -
              misfit_t((t0s[0] - eps * v[0], t0s[1] - eps * v[1]))) / (2 * eps)
        tfd.append(abs(fd - dot((tgre, tgim), v)) / abs(fd))
    o = Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], dt=c["dt"], bc_mode=tbc)
    for k, (a, b) in state.items():
        o.set_field(k, a, b)
    o.set_field("temp", *t0s)
    o.step(c["steps"])
    tresid = o.synth_scalar(*o.get_field("temp"))[mid] - tgt
    o = Oracle(lmax=c["lmax"], nlat=c["nlat"], nlon=c["nlon"], nr=c["nr"], dt=c["dt"], bc_mode=tbc)
    for k, (a, b) in state.items():
        o.set_field(k, a, b)
    o.set_field("temp", *tdirs[0])  # the tangent: zero sources and boundary values
    o.step(c["steps"])
    tfm = float(np.sum(tresid * o.synth_scalar(*o.get_field("temp"))[mid]))
    temperature = {"objective": "1/2 |T(r_mid) - target|^2 after the steps, w.r.t. the initial temperature",
                   "bc_mode": tbc,
                   "J": JT, "fd_rel_err_max": max(tfd), "fd_directions": len(tfd),
                   "oracle_forward_mode_rel_err": abs(tfm - dot((tgre, tgim), tdirs[0])) / abs(tfm),
                   "misfit_and_gradient_s_wall": t_temp,
                   "reverse": "velocity grids recomputed per 20-step segment from device snapshots"}
    line = {"metric": "adjoint gradient vs FP64 finite differences (max relative error, 32 directions)",
            "value": max(fd_err), "unit": "relative error", "higher_is_better": False, "n_gpus": 1,
            "dtype": "f64", "data": "synthetic (adjoint_state(0): seeded_state(0) with zero temperature; adjoint_target(seed=1); directions default_rng(2))",
            "config": {"workload": "adjoint_l63_nr65", "lmax": c["lmax"], "nlat": c["nlat"], "nlon": c["nlon"],
                       "nr": c["nr"], "steps": c["steps"], "dt": c["dt"], "bc_mode": c["bc_mode"],
                       "checkpoint_every": c["checkpoint"]},
            "J": J, "fd_rel_err_max": max(fd_err), "fd_rel_err_median": float(np.median(fd_err)),
            "oracle_forward_mode_rel_err_max": max(fm_err), "forward_ms_device": fwd_ms,
            "pullback_ms_wall": pull_ms, "misfit_and_gradient_s_wall": t_total, "checkpoints": len(ckpt),
            "temperature": temperature}
    print(json.dumps(line), flush=True)
    return 0


def run_accuracy_study(args, gdb, workloads, torch):
    """The headline condition's error budget at the headline workload: kinetic
    and magnetic energy relative errors after 100 and 1000 steps of
    (1) the FP64 step started from the seeded state perturbed by one ulp in
        every coefficient, against the unperturbed FP64 step (the floor any
        implementation meets), under the literal operator (bc_mode 0) and with
        Dirichlet rows (bc_mode 2);
    (2) the mixed step with no stage, each single stage and all stages of the
        velocity chain returned to FP64 (gd_set_fp64_stages), against the FP64
        step, with each configuration's device time per step."""
    p = workload_params()
    st = workloads.seeded_state(p["lmax"], p["lmax"], p["nr"], seed=0)
    marks = (100, args.accuracy_steps)

    def make(prec, bc, state):
        g = gdb.SHTnsKitConfig(p["lmax"], p["nlat"], p["nlon"], p["nr"], dt=p["dt"], rratio=p["rratio"],
                               ekman=p["ekman"], rayleigh=p["rayleigh"], prandtl=p["prandtl"],
                               magnetic_prandtl=p["magnetic_prandtl"], implicit_theta=p["implicit_theta"],
                               bc_mode=bc, precision=prec)
        for k, (a, b) in state.items():
            g.set_field(k, a, b)
        return g

    def trajectory(g):
        out, done = [], 0
        for m in marks:
            g.step(m - done)
            done = m
            out.append(g.energy())
        return out

    def rel_err(x, y):
        return {f"{n}_rel_err_{m}": abs(a[i] - b[i]) / abs(b[i])
                for i, n in enumerate(("ekin", "emag")) for m, a, b in zip(marks, x, y)}

    def ms_per_step(g, n=10):
        ext = torch.cuda.ExternalStream(g.stream_ptr())
        g.step(3)
        g.synchronize()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext); g.step_async(n); e1.record(ext); e1.synchronize(); g.synchronize()
        return e0.elapsed_time(e1) / n

    pert = {k: (np.nextafter(a, np.inf), np.nextafter(b, np.inf)) for k, (a, b) in st.items()}
    res = {"steps": list(marks), "floor": {}, "budget": {}}
    for bc in (0, 2):
        g = make("fp64", bc, st)
        ref = trajectory(g)
        if bc == 2:
            res["fp64_ms_per_step"] = ms_per_step(g)
        g.close()
        g = make("fp64", bc, pert)
        res["floor"][f"bc{bc}"] = rel_err(trajectory(g), ref)
        g.close()
        rows = ([(), ("vel_synth",), ("vel_products",), ("vel_analysis",), ("vel_synth", "vel_products", "vel_analysis")]
                if bc == 2 else [(), ("vel_synth", "vel_products", "vel_analysis")])
        for stages in rows:
            g = make("mixed", bc, st)
            g.set_fp64_stages(stages)
            row = rel_err(trajectory(g), ref)
            if bc == 2:
                row["ms_per_step"] = ms_per_step(g)
            res["budget"][f"bc{bc}:" + ("+".join(stages) or "none")] = row
            g.close()
    line = {"metric": "energy error budget of the mixed step (relative to the FP64 step)", "value": None,
            "unit": "relative error", "n_gpus": 1, "higher_is_better": False,
            "data": "synthetic (seeded default_rng(0) state, amplitude 1e-3 (l+1)^-2)",
            "config": {"workload": WORKLOAD, "lmax": p["lmax"], "nlat": p["nlat"], "nlon": p["nlon"], "nr": p["nr"],
                       "dt": p["dt"]}, **res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed", "mixed_vel64", "mixed_vel64i8"],
                    help="auto: mixed_vel64i8 (the mixed step with its velocity chain at FP64 accuracy, its "
                         "synthesis by int8 digit slices on the tensor cores: the configuration that meets the energy "
                         "condition) when the device has tcgen05, else fp64")
    ap.add_argument("--accuracy-study", action="store_true",
                    help="instead of the headline: the FP64 one-ulp floor and the per-stage error budget")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the FP64 vs mixed energy comparison (0 = skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD,
                    help="named shell workload (the headline metric is shell_l255_nr129; smaller ones are for profiling)")
    ap.add_argument("--transforms", action="store_true",
                    help="instead of the headline: the transform-only batch's errors and timings")
    ap.add_argument("--adjoint", action="store_true",
                    help="instead of the headline: the adjoint configuration's gradient checks and timings")
    ap.add_argument("--ensemble-group", type=int, default=64,
                    help="ensemble: members of one lmax per segmented handle, at most this many (1: a handle each)")
    ap.add_argument("--ensemble", type=int, default=0,
                    help="instead of the headline: the batched uneven ensemble of this many shells")
    ap.add_argument("--decomposed", action="store_true",
                    help="one model across the ranks (mode/shell decomposition, NCCL all-to-alls)")
    ap.add_argument("--scheme", default="cnab2", choices=["cnab2", "eab2", "erk2"],
                    help="time-stepping scheme of the step (ts_scheme); the headline metric is CNAB2")
    args = ap.parse_args()
    if args.workload != WORKLOAD:
        globals()["WORKLOAD"] = args.workload
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    gdb = load_package()
    import workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.ensemble > 0:
        return run_ensemble(args, gdb, workloads, torch, world, rank)
    if args.decomposed:
        return run_decomposed(args, gdb, workloads, torch, world, rank, local)
    if args.adjoint:
        return run_adjoint(args, gdb, workloads, torch)
    if args.transforms:
        return run_transforms(args, gdb, workloads, torch)
    if args.accuracy_study:
        return run_accuracy_study(args, gdb, workloads, torch)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    p = workload_params()
    st = workloads.seeded_state(p["lmax"], p["lmax"], p["nr"], seed=0)

    def make(precision, bc_mode=0):
        g = gdb.SHTnsKitConfig(p["lmax"], p["nlat"], p["nlon"], p["nr"], dt=p["dt"], rratio=p["rratio"],
                               ekman=p["ekman"], rayleigh=p["rayleigh"], prandtl=p["prandtl"],
                               magnetic_prandtl=p["magnetic_prandtl"], implicit_theta=p["implicit_theta"],
                               bc_mode=bc_mode, precision="fp64", device=local)
        if precision != "fp64":
            g.set_precision(precision)
        if args.scheme != "cnab2" and bc_mode != 2:
            g.set_scheme(args.scheme)
        for k, (a, b) in st.items():
            g.set_field(k, a, b)
        return g

    precision = args.precision
    if precision == "auto":
        try:
            probe = gdb.SHTnsKitConfig(7, 12, 24, 9, device=local)
            probe.set_precision("mixed")
            probe.close()
            precision = "mixed_vel64i8"
        except gdb.GeoDynamoError:
            precision = "fp64"

    def timed_steps(g, K, W):
        ext = torch.cuda.ExternalStream(g.stream_ptr())
        g.step(W)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        g.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        g.step_async(K)
        e1.record(ext)
        e1.synchronize()
        g.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- main timed region ----
    g = make(precision)
    clocks = ClockSampler(local)
    g.step(args.warmup)
    clocks.start()
    ms_total = timed_steps(g, args.steps, 0)
    clk = clocks.stop()
    value = world * args.steps / (ms_total / 1e3)
    ms_per_step = ms_total / args.steps

    # ---- per-kernel breakdown (events around each launch, eager replay) ----
    nprof = 2

    def breakdown(h, prec):
        h.profile_enable(True)
        h.step(nprof)
        pr = h.profile_read()
        h.profile_enable(False)
        out = []
        for name, (ms, cnt) in sorted(pr.items(), key=lambda kv: -kv[1][0]):
            per = ms / cnt
            w = kernel_work(name, p, h.nlm, prec)
            ent = {"name": name, "share": None, "launches_per_step": cnt / nprof, "ms_per_launch": per}
            if name.startswith("fft_"):
                # 4-component synth launches and 2-component ones share a name; use the per-step mix
                if prec == "fp64":
                    ncomp = (4 + 2 * 4) if "synth" in name else (1 + 2 + 2)
                else:  # the FP64 velocity stages of the mixed step: u (synthesis), its products (analysis)
                    ncomp = 2
                ent["gbs"] = fft_bytes(p, ncomp, prec) / (ms / nprof / 1e3) / 1e9
            elif w is not None:
                if w["flops"] is not None:
                    ent["tflops"] = w["flops"] / (per / 1e3) / 1e12
                if w["bytes"] is not None:
                    ent["gbs"] = w["bytes"] / (per / 1e3) / 1e9
            out.append(ent)
        tot = sum(v[0] for v in pr.values())
        for ent in out:
            ent["share"] = pr[ent["name"]][0] / tot if tot else None
        return pr, out

    prof, kernels = breakdown(g, precision)
    dgemm = fp64_gemm_tflops()

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    top = kernels[0] if kernels else None
    roofline = None
    if top is not None:
        bounds = []
        if "gbs" in top:
            bounds.append({"bound": "hbm", "achieved": top["gbs"], "peak": hbm_peak, "unit": "GB/s",
                           "frac": top["gbs"] / hbm_peak, "peak_source": peak_src + " HBM copy bandwidth"})
        if "tflops" in top:
            if top["name"].endswith("fp64") or top["name"].startswith(("eab2", "erk2")):
                pk, src = dgemm, "cuBLAS FP64 GEMM 4096^3 measured in this run (torch.matmul)"
            elif top["name"].endswith("_i8"):
                pk, src = peaks.get("bf16_tflops", 1590.0) * 2.0, "twice the measured bf16 burst peak (int8 rate)"
            else:
                pk, src = peaks.get("bf16_tflops", 1590.0) / 2.0, "half the measured bf16 burst peak (tf32 rate)"
            bounds.append({"bound": "tensor", "achieved": top["tflops"], "peak": pk, "unit": "TFLOP/s",
                           "frac": top["tflops"] / pk, "peak_source": src})
        if bounds:
            bounds.sort(key=lambda b: -b["frac"])  # the binding roof is the one closest to its limit
            roofline = dict(bounds[0])
            roofline["kernel"] = top["name"]
            roofline["traffic"] = measured_traffic(top["name"])
            roofline["traffic_unit"] = "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)"
            if len(bounds) > 1:
                roofline["other"] = {k: bounds[1][k] for k in ("bound", "achieved", "peak", "unit", "frac")}
            if top["name"].startswith("fused_"):
                # what does bind the fused phase kernels (one-launch ncu capture at nr = 33,
                # profiles/fused_velocity_fp32_shell_l255_nr33.md): neither HBM nor a tensor pipe
                roofline["binding_unit"] = {"unit": "shared-memory (LSU) wavefronts and issue",
                                            "lsu_frac": 0.61, "issue_active_frac": 0.58,
                                            "source": "ncu, k_fused<768, 2, 0>, shell_l255_nr33"}

    # ---- FP64 reference step on the GPU (denominator of the metric) ----
    fp64_value = None
    k64 = kernels
    if precision != "fp64":
        g64 = make("fp64")
        g64.step(args.warmup)
        ms64 = timed_steps(g64, args.steps, 0)
        fp64_value = world * args.steps / (ms64 / 1e3)
        _, k64 = breakdown(g64, "fp64")
        g64.close()
    else:
        fp64_value = value
    # how tuned the denominator is: the FP64 step's Legendre contractions
    # (DMMA) against the measured cuBLAS FP64 GEMM rate
    leg = [k for k in k64 if k["name"].startswith("legendre_") and "tflops" in k]
    leg_ms = sum(k["ms_per_launch"] * k["launches_per_step"] for k in leg)
    leg_tf = sum(k["tflops"] * k["ms_per_launch"] * k["launches_per_step"] for k in leg)
    fp64_den = {"ms_per_step": 1e3 / (fp64_value / world) if fp64_value else None,
                "legendre_ms_per_step": leg_ms,
                "legendre_tflops": leg_tf / leg_ms if leg_ms else None,
                "fp64_gemm_tflops": dgemm,
                "legendre_frac_of_gemm": leg_tf / leg_ms / dgemm if leg_ms else None}

    # ---- energy agreement, mixed vs FP64 ----
    # bc_mode 0 is the reference's operator as written (no boundary rows; its
    # temperature grows without bound at nr = 129, dt = 2e-6 in FP64 too);
    # bc_mode 2 adds Dirichlet rows to the implicit operator.
    # the fast mixed step (every stage in mixed precision) beside the headline
    # configuration, when the headline is the one with its velocity chain in FP64
    variants = {}
    if precision in ("mixed_vel64", "mixed_vel64i8"):
        gf = make("mixed")
        gf.step(args.warmup)
        msf = timed_steps(gf, args.steps, 0)
        variants["mixed"] = {"value": world * args.steps / (msf / 1e3), "unit": "steps/s",
                             "ms_per_step": msf / args.steps,
                             "ratio_vs_fp64_gpu": world * args.steps / (msf / 1e3) / fp64_value,
                             "what": "every transform and product in split-TF32 / FP32"}
        gf.close()
    accuracy = None
    if precision != "fp64" and args.accuracy_steps > 0:
        accuracy = {"steps": args.accuracy_steps, "target_rel_err": 1e-9}
        for label, bc in (("literal_bc0", 0), ("dirichlet_bc2", 2)):
            gb = make("fp64", bc)
            gb.step(args.accuracy_steps)
            eb = gb.energy()
            gb.close()
            accuracy[label] = {"ekin_fp64": eb[0], "emag_fp64": eb[1]}
            for v in [precision] + list(variants):
                ga = make(v, bc)
                ga.step(args.accuracy_steps)
                ea = ga.energy()
                ga.close()
                accuracy[label][v] = {"ekin_rel_err": abs(ea[0] - eb[0]) / abs(eb[0]),
                                      "emag_rel_err": abs(ea[1] - eb[1]) / abs(eb[1])}
        for v in variants:
            variants[v]["accuracy_dirichlet_bc2"] = accuracy["dirichlet_bc2"][v]

    # ---- end to end through the C ABI with host buffers ----
    names = list(workloads.FIELD_ORDER)
    pinned = {}
    for k in names:
        a, b = st[k]
        ta = torch.from_numpy(a).pin_memory()
        tb = torch.from_numpy(b).pin_memory()
        pinned[k] = (ta, tb)
    out_pinned = {k: (torch.empty(st[k][0].shape, dtype=torch.float64).pin_memory(),
                      torch.empty(st[k][1].shape, dtype=torch.float64).pin_memory()) for k in names}
    import ctypes
    lib = g.lib
    D = ctypes.POINTER(ctypes.c_double)
    ptr = lambda t: ctypes.cast(t.data_ptr(), D)  # noqa: E731
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in names:
        g._check(lib.gd_upload_spectral(g.h, gdb.FIELDS[k], ptr(pinned[k][0]), ptr(pinned[k][1])))
    energies = []
    for _ in range(args.steps):
        # every step: one graph step and its result (the two energies) read back
        g.step_async(1)
        energies.append(g.energy())
    for k in names:
        g._check(lib.gd_download_spectral(g.h, gdb.FIELDS[k], ptr(out_pinned[k][0]), ptr(out_pinned[k][1])))
    e2e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    state_bytes = sum(a.nbytes + b.nbytes for a, b in st.values())
    e2e = {"value": world * args.steps / e2e_s, "unit": "steps/s",
           "h2d_bytes_per_step": state_bytes / args.steps, "d2h_bytes_per_step": 16 + state_bytes / args.steps,
           "job": f"upload 5 fields from pinned host memory, {args.steps} graph steps each followed by a read of "
                  f"its energies, 5 fields back"}

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, dts, cores = cpu_reference_rate(1, 1)
        cpu = {"value": rate, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": f"oracle at the full {WORKLOAD} grid (lmax={p['lmax']} nlat={p['nlat']} nlon={p['nlon']} "
                         f"nr={p['nr']}), 1 timed step after 1 warm-up on {cores} threads ({dts:.2f} s); the "
                         f"one-thread figure is in the reference arm's line"}

    gpu_launches = g.step_kernels() * args.steps  # kernel nodes of the step graph x timed steps
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None,
                "dtype": {"fp64": "f64", "mixed": "f32/tf32x3 (FP64 solves)",
                          "mixed_vel64": "f32/tf32x3, velocity chain f64 (FP64 solves)",
                          "mixed_vel64i8": "f32/tf32x3, velocity chain f64 with its synthesis in int8 "
                                           "digit slices (FP64 solves)"}[precision],
                "data": "synthetic (seeded default_rng(0) state, amplitude 1e-3 (l+1)^-2)",
                "config": {"workload": WORKLOAD, "lmax": p["lmax"], "nlat": p["nlat"], "nlon": p["nlon"], "nr": p["nr"],
                           "dt": p["dt"], "precision": precision, "parallelism": f"replicas x{world}",
                           "l2": "working set 5+ GB of grids per step, larger than L2; no flush"},
                "fp64_gpu_value": fp64_value, "ratio_vs_fp64_gpu": value / fp64_value if fp64_value else None,
                "fp64_denominator": fp64_den, "variants": variants,
                "fp64_kernels": k64 if precision != "fp64" else None,
                "accuracy": accuracy, "roofline": roofline, "kernels": kernels, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": gpu_launches, "clocks": clk}
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
