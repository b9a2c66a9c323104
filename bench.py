#!/usr/bin/env python
"""Benchmark: LJ MD (FP64 plain GPU path) on the 4,096,000-particle workload.

Workload: 160^3 simple-cubic lattice at spacing 1.1 sigma (+-0.05 jitter), periodic
176^3 box, eps = sigma = 1, r_cut = 2.5, Verlet list with skin 0.3 rebuilt when
the largest displacement exceeds skin/2, velocity Verlet dt = 0.005, Gaussian
velocities at T = 1.  One step = one velocity-Verlet step of the whole system
(integrate, image refresh or rebuild, forces).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  Multi-GPU: the path does not shard (one GPU per system),
so N ranks run N independent replicas ("replicas only"); value sums them and
the time is the max over ranks.
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

METRIC = "particle-steps/s"
N_SIDE, SPACING, JITTER, SEED = 160, 1.1, 0.05, 2
R_CUT, SKIN, DT, EPS, SIGMA, MASS = 2.5, 0.3, 0.005, 1.0, 1.0, 1.0
WORKLOAD = "LJ MD 3D FP64, N=4,096,000 (160^3 lattice, spacing 1.1, jitter 0.05), box 176, r_cut 2.5, " \
           "Verlet skin 0.3 (rebuild at max displacement > skin/2), velocity Verlet dt 0.005"


def workload_name(nside, mixed):
    w = WORKLOAD if not mixed else WORKLOAD.replace("FP64", "mixed-precision")
    if nside != N_SIDE:
        w = w.replace("N=4,096,000 (160^3", f"N={nside ** 3:,} ({nside}^3").replace(
            "box 176", f"box {nside * SPACING:g}") + " [profiling case]"
    return w


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(kernel_file, key="traffic_bytes_per_launch"):
    """dram bytes per force launch (scaled to the full workload) from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", kernel_file)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(nside=N_SIDE):
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(nside, SPACING, JITTER, seed=SEED)
    return x, v, L


TUNE = {"tiles": 1, "tx": 0, "tpp": 0, "precision": "fp64"}


def build_system(pd, x, v, L):
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    mixed = TUNE["precision"] == "mixed"
    pt = pd.PD_F32 if mixed else pd.PD_F64
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, R_CUT + SKIN, dtype=np.float64, props=[(pt, 3), (pt, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=DT, mass=MASS, skin=SKIN, eps=EPS, sigma=SIGMA, r_cut=R_CUT,
               precision=pd.PREC_MIXED if mixed else pd.PREC_FP64)
    md.set_tiles(bool(TUNE["tiles"]), TUNE["tx"], TUNE["tpp"])
    return vd, md


def cpu_reference(x, v, L, steps, budget_s=30.0):
    """The oracle's FP64 velocity-Verlet loop on this host's cores (all threads)."""
    from oracle import pyoracle as orc
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    threads = orc.num_threads()
    # probe one step to size the bounded sample
    _, _, _, t1 = orc.md_lj(x, v, lo, hi, bc, R_CUT + SKIN, R_CUT, SKIN, EPS, SIGMA, DT, MASS, 1, timing=True)
    k = int(max(2, min(steps, budget_s / max(t1, 1e-3))))
    _, _, E, t = orc.md_lj(x, v, lo, hi, bc, R_CUT + SKIN, R_CUT, SKIN, EPS, SIGMA, DT, MASS, k, timing=True)
    rebuilds = int(E[1:, 3].sum())
    return x.shape[0] * k / t, threads, k, rebuilds, t


def reference_arm(steps, warmup, budget_s=240.0):
    """--impl reference: the oracle's FP64 loop (the reference's CPU algorithm restated;
    its own CPU path cannot be compiled here) on all host threads, W untimed warm-up
    steps and then exactly K timed steps of the full 4,096,000-particle system; when
    K steps would exceed the budget, every step runs on a bounded sample instead: a
    smaller lattice of the same spacing, density and jitter, whose particle-steps/s
    is the rate reported.  Returns (value, threads, particles, rebuilds, seconds)."""
    from oracle import pyoracle as orc
    threads = orc.num_threads()
    nside = N_SIDE
    x, v, L = make_workload(nside)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    _, _, _, t1 = orc.md_lj(x, v, lo, hi, bc, R_CUT + SKIN, R_CUT, SKIN, EPS, SIGMA, DT, MASS, 1, timing=True)
    if (steps + warmup) * t1 > budget_s:
        nside = max(24, int(nside * (budget_s / ((steps + warmup) * t1)) ** (1.0 / 3.0)))
        x, v, L = make_workload(nside)
        lo, hi = np.zeros(3), np.full(3, L)
    xw, vw = x, v
    if warmup > 0:
        xw, vw, _ = orc.md_lj(x, v, lo, hi, bc, R_CUT + SKIN, R_CUT, SKIN, EPS, SIGMA, DT, MASS, warmup)
    _, _, E, t = orc.md_lj(xw, vw, lo, hi, bc, R_CUT + SKIN, R_CUT, SKIN, EPS, SIGMA, DT, MASS, steps, timing=True)
    return x.shape[0] * steps / t, threads, x.shape[0], int(E[1:, 3].sum()), t


def bench_config(n, world, nside=N_SIDE, mixed=False):
    """The workload description both arms print (run-dependent list statistics are reported apart)."""
    return {"workload": workload_name(nside, mixed), "particles": n,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (positions 131 MB + Verlet list ~1.1 GB per replica)"}


def _timed(md, steps, torch):
    """Run `steps` steps between two CUDA events on torch's current stream (the library's
    launches go to the legacy default stream, which synchronises with it); returns (ms, E)."""
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    E = md.run(steps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), E


def form_precision(pd, torch, x, v, L, steps, warmup, fp64_value):
    """Precision form on the 4,096,000-particle lattice: throughput, ratio to the FP64
    path and the force error against the FP64 GPU path on the final positions."""
    TUNE["precision"] = "mixed"
    vd, md = build_system(pd, x, v, L)
    md.run(warmup, energies=False)
    md.set_timing(True)
    ms, E = _timed(md, steps, torch)
    t = md.timers()
    n = x.shape[0]
    val = n * steps / (ms / 1e3)
    # forces of the FP64 path on the same (final) positions
    xf = vd.deviceToHostPos(with_ghost=False)
    f32 = vd.deviceToHostProp(1, with_ghost=False).astype(np.float64)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd64 = pd.VectorDist(n, lo, hi, bc, R_CUT, dtype=np.float64, props=[(pd.PD_F64, 3)])
    vd64.hostToDevicePos(xf)
    vd64.map()
    vd64.ghost_get()
    cl = vd64.getCellListGPU(R_CUT)
    vd64.updateCellListGPU(cl)
    vd64.lj_forces(0, cl=cl, eps=EPS, sigma=SIGMA, r_cut=R_CUT)
    f64 = vd64.deviceToHostProp(0, with_ghost=False)  # same order as xf (map on one domain keeps it)
    frms = np.sqrt((f64 ** 2).sum(axis=1).mean())
    err = np.sqrt(((f32 - f64) ** 2).sum(axis=1)) / frms
    gerr = float(np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum()))
    TUNE["precision"] = "fp64"
    return {"workload": workload_name(N_SIDE, True), "value": val, "unit": METRIC, "steps": steps,
            "ms_per_step": ms / steps, "vs_fp64_path": val / fp64_value,
            "phases_ms_per_step": {k: (tv[0] / max(tv[1], 1)) for k, tv in t.items()},
            "list_rebuilds": int(E[:, 3].sum()),
            "force_error_vs_fp64": {"mean": float(err.mean()), "max": float(err.max()), "global": gerr,
                                    "norm": "per particle |F32 - F64| / F_rms(F64) at the final positions; "
                                            "global = ||F32 - F64|| / ||F64||"}}


def fp64_forces(pd, x, L):
    """LJ forces of the FP64 GPU cell-list path (the path the parity tests hold to
    the FP64 oracle) at positions x, in the order of x."""
    n = x.shape[0]
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(n, lo, hi, bc, R_CUT, dtype=np.float64, props=[(pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.map()
    vd.ghost_get()
    cl = vd.getCellListGPU(R_CUT)
    vd.updateCellListGPU(cl)
    vd.lj_forces(0, cl=cl, eps=EPS, sigma=SIGMA, r_cut=R_CUT)
    f = vd.deviceToHostProp(0, with_ghost=False)
    del cl, vd
    return f


def form_clustered(pd, torch, steps=200, check_every=20, warmup=3):
    """Precision form on the clustered layout: 4,096,000 particles in 64 Gaussian
    clusters (sigma_c 8) at uniform centres in a 176 periodic box, minimum distance
    0.8 (redraws, then centre moves); force error against the FP64 path every
    `check_every` steps."""
    from openfpm_pdata_b200 import workloads
    t0 = time.perf_counter()
    x, v, L, redraws = workloads.lj_clustered_lib(4096000, 176.0, seed=4)
    t_gen = time.perf_counter() - t0
    n = x.shape[0]
    TUNE["precision"] = "mixed"
    vd, md = build_system(pd, x, v, L)
    TUNE["precision"] = "fp64"
    md.run(warmup, energies=False)
    errs, ms_tot, done, rebuilds = [], 0.0, 0, 0
    while done < steps:
        k = min(check_every, steps - done)
        ms, E = _timed(md, k, torch)
        ms_tot += ms
        done += k
        rebuilds += int(E[:, 3].sum())
        xf = vd.deviceToHostPos(with_ghost=False)
        f32 = vd.deviceToHostProp(1, with_ghost=False).astype(np.float64)
        f64 = fp64_forces(pd, xf, L)
        frms = np.sqrt((f64 ** 2).sum(axis=1).mean())
        e = np.sqrt(((f32 - f64) ** 2).sum(axis=1)) / frms
        g = np.sqrt(((f32 - f64) ** 2).sum() / (f64 ** 2).sum())
        errs.append((done, float(e.mean()), float(e.max()), float(g)))
    cnt = np.bincount((np.floor(x / (L / 62)).astype(int) % 62) @ np.array([1, 62, 62 * 62]), minlength=62 ** 3)
    del md, vd
    return {"workload": "LJ MD mixed-precision, N=4,096,000 in 64 Gaussian clusters (sigma_c 8) at uniform "
                        "centres, periodic box 176, minimum distance 0.8, r_cut 2.5, skin 0.3, dt 0.005",
            "value": n * steps / (ms_tot / 1e3), "unit": METRIC, "steps": steps, "ms_per_step": ms_tot / steps,
            "list_rebuilds": rebuilds, "generator_s": t_gen, "centre_redraws": redraws,
            "layout": {"cell_occupancy_max": int(cnt.max()), "cell_occupancy_p99": float(np.percentile(cnt, 99)),
                       "cell_occupancy_mean": float(cnt.mean()), "cell_side": L / 62},
            "force_error_vs_fp64": {"steps_checked": [e[0] for e in errs],
                                    "mean": [e[1] for e in errs], "max": [e[2] for e in errs],
                                    "global": [e[3] for e in errs],
                                    "norm": "per particle |F32 - F64| / F_rms(F64); global = ||F32 - F64|| / ||F64||"}}


def form_cell_list_every_step(pd, torch, steps=100, warmup=5):
    """N = 4096 (16^3 lattice, spacing 1, box 16), cell list rebuilt every step, FP64."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(16, 1.0, 0.05, seed=1)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(x.shape[0], lo, hi, bc, R_CUT, dtype=np.float64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, v)
    md = pd.MD(vd, 0, 1, dt=DT, mass=MASS, skin=0.0, eps=EPS, sigma=SIGMA, r_cut=R_CUT, use_cell_list=True)
    md.run(warmup, energies=False)
    l0 = pd.launch_count()
    ms, E = _timed(md, steps, torch)
    return {"workload": "LJ MD FP64, N=4096 (16^3 lattice, spacing 1, jitter 0.05), box 16, r_cut 2.5, "
                        "cell list rebuilt every step, dt 0.005",
            "value": x.shape[0] * steps / (ms / 1e3), "unit": METRIC, "steps": steps, "ms_per_step": ms / steps,
            "gpu_launches_per_step": (pd.launch_count() - l0) / steps,
            "cluster_ctas": md.launch_shape()["cluster_ctas"]}


def _ev_ms(torch, fn, reps):
    """Mean ms of `fn` over `reps` calls between CUDA events (the calls synchronise themselves)."""
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def form_symmetric(pd, torch, x, L, reps=20):
    """LJ forces on the 4,096,000-particle lattice from global-index rows: the full
    Verlet list against the symmetric (half) list with reactions on the partners
    and ghost_put<add_> folding the ghosts' share (FP64)."""
    n = x.shape[0]
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(n, lo, hi, bc, R_CUT + SKIN, dtype=np.float64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    vd.hostToDevicePos(x)
    vd.map()
    vd.ghost_get()
    rl = R_CUT + SKIN
    full = vd.getVerlet(rl)
    half = vd.getVerletSym(rl)
    t_full_build = _ev_ms(torch, lambda: vd.updateVerlet(full), 3)
    t_half_build = _ev_ms(torch, lambda: vd.updateVerlet(half), 3)
    f_full = lambda: vd.lj_forces(0, vl=full, eps=EPS, sigma=SIGMA, r_cut=R_CUT)

    def f_half():
        vd.lj_forces(1, vl=half, eps=EPS, sigma=SIGMA, r_cut=R_CUT)
        vd.ghost_put([1])
    f_full()
    f_half()
    t_full = _ev_ms(torch, f_full, reps)
    t_half = _ev_ms(torch, f_half, reps)
    a = vd.deviceToHostProp(0, with_ghost=False)
    b = vd.deviceToHostProp(1, with_ghost=False)
    frms = np.sqrt((a ** 2).sum(axis=1).mean())
    off, _ = full.get()
    hoff, _ = half.get()
    del full, half, vd
    return {"workload": "LJ forces FP64, N=4,096,000 lattice (spacing 1.1), r_cut 2.5, list radius 2.8, "
                        "global-index rows",
            "full_list": {"ms": t_full, "entries": int(off[-1]), "build_ms": t_full_build},
            "half_list_plus_ghost_put": {"ms": t_half, "entries": int(hoff[-1]), "build_ms": t_half_build},
            "max_force_diff_over_frms": float(np.abs(a - b).max() / frms)}


def form_compaction(pd, torch, n=4096000, frac=0.1, reps=5):
    """remove_marked and get_indexes_by_type on 4,096,000 FP64 particles with two
    3-component FP64 properties and an int mark (10 % marked)."""
    rng = np.random.default_rng(21)
    L = 176.0
    x = rng.uniform(0, L, size=(n, 3))
    v = rng.normal(size=(n, 3))
    mark = (rng.random(n) < frac).astype(np.int32)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    vd = pd.VectorDist(n, lo, hi, bc, 1.0, dtype=np.float64,
                       props=[(pd.PD_F64, 3), (pd.PD_F64, 3), (pd.PD_I32, 1)])
    t_rm, t_ix = [], []
    kept = 0
    for it in range(reps + 1):
        vd.resize(n)
        vd.hostToDevicePos(x)
        vd.hostToDeviceProp(0, v)
        vd.hostToDeviceProp(1, v)
        vd.hostToDeviceProp(2, mark)
        t_ix.append(_ev_ms(torch, lambda: vd.get_indexes_by_type(2, 1, device=True), 1))
        t_rm.append(_ev_ms(torch, lambda: vd.remove_marked(2), 1))
        kept = vd.size_local()
    t_rm, t_ix = float(np.mean(t_rm[1:])), float(np.mean(t_ix[1:]))
    rec = 32 + 4 + 3 * 8 * 2 + 4  # position record, global id, two FP64 vectors, the mark
    alg = n * rec + kept * rec
    hbm, which = peaks()
    del vd
    return {"workload": "remove_marked / get_indexes_by_type, N=4,096,000 FP64 particles, props "
                        "double[3], double[3], int mark, 10% marked",
            "remove_marked_ms": t_rm, "kept": kept,
            "remove_marked_roofline": {"bound": "hbm", "algorithmic_bytes": alg,
                                       "achieved_gbs": alg / (t_rm / 1e3) / 1e9, "peak_gbs": hbm,
                                       "frac": alg / (t_rm / 1e3) / 1e9 / hbm, "peak_kind": which,
                                       "bytes": "read every record once, write every kept record once"},
            "get_indexes_by_type_ms": t_ix,
            "note": "both calls include their device-to-host count read and synchronise; the indexes "
                    "stay in device memory"}


def form_sph(pd, torch, steps=200, warmup=5, dp=1.0 / 180):
    """WCSPH dam break, FP64 and FP32 storage."""
    from openfpm_pdata_b200 import workloads
    x, typ, m, lo, hi = workloads.sph_dam(dp)
    h = 1.3 * dp
    out = {"workload": f"WCSPH dam break, fluid block [0,0.4]x[0,1]x[0,0.6] + 3 wall layers, dp=1/{round(1 / dp)}, "
                       f"N={x.shape[0]:,}, h=1.3dp, c0=20, rho0=1000, alpha=0.1, dt=1e-4, Verlet skin 0.3dp",
           "particles": int(x.shape[0])}
    for name, dt_ in (("fp64", np.float64), ("fp32", np.float32)):
        ft = pd.PD_F64 if dt_ == np.float64 else pd.PD_F32
        vd = pd.VectorDist(x.shape[0], lo, hi, np.zeros(3, np.int32), 0.0, dtype=dt_,
                           props=[(ft, 3), (ft, 3), (ft, 1), (ft, 1), (pd.PD_I32, 1)])
        vd.hostToDevicePos(x.astype(dt_))
        vd.hostToDeviceProp(0, np.zeros((x.shape[0], 3)))
        vd.hostToDeviceProp(2, np.full(x.shape[0], 1000.0))
        vd.hostToDeviceProp(4, typ)
        sph = pd.SPH(vd, 0, 1, 2, 3, 4, h, m, 20.0, 1000.0, 0.1, -9.81, 1e-4, skin=0.3 * dp)
        sph.run(warmup, energies=False)
        sph.set_timing(True)
        ms, E = _timed(sph, steps, torch)
        t = sph.timers()
        out[name] = {"value": x.shape[0] * steps / (ms / 1e3), "unit": METRIC, "steps": steps,
                     "ms_per_step": ms / steps, "list_rebuilds": int(E[:, 3].sum()),
                     "phases_ms_per_step": {k: (tv[0] / max(tv[1], 1)) for k, tv in t.items()}}
        del sph, vd
    return out


def form_serving(pd, torch, n_systems=600, steps=50, slots=128, seed=6, loads=(0.4, 0.6, 0.8)):
    """Serving form: a bounded sample of the stream of independent LJ systems
    (N log-uniform in [512, 262144], density 0.8, 50 steps each).
    (1) capacity: a quarter of the sample submitted at once;
    (2) Poisson arrivals at `loads` x that capacity (a quarter of the sample each):
        p50/p99 latency (arrival -> result) and aggregate throughput;
    (3) isolated (measured first): systems run one after another through the
        single-system driver."""
    from openfpm_pdata_b200 import workloads
    sizes = workloads.serving_sizes(n_systems, seed=seed)
    systems = [workloads.serving_system(int(n), 0.8, seed=1000 + k) for k, n in enumerate(sizes)]
    part = n_systems // (1 + len(loads))
    # (3) isolated, measured first (before the server holds its pool): the
    # single-system mixed-precision driver, one system after another; one
    # untimed system first loads the driver's kernels

    def run_isolated(x, v, L):
        vd = pd.VectorDist(x.shape[0], np.zeros(3), np.full(3, L), np.ones(3, np.int32), R_CUT + SKIN,
                           dtype=np.float64, props=[(pd.PD_F32, 3), (pd.PD_F32, 3)])
        vd.hostToDevicePos(x)
        vd.hostToDeviceProp(0, v)
        md = pd.MD(vd, 0, 1, dt=DT, skin=SKIN, precision=pd.PREC_MIXED)
        md.run(steps)
        vd.deviceToHostPos(with_ghost=False)
        del md, vd
    sub = systems[part: part + 40]
    run_isolated(*systems[-1])
    plain_lat, plain_ps = [], 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for (x, v, L) in sub:
        t1 = time.perf_counter()
        run_isolated(x, v, L)
        plain_lat.append(time.perf_counter() - t1)
        plain_ps += x.shape[0] * steps
    t_plain = time.perf_counter() - t0
    iso = plain_ps / t_plain
    free, _ = torch.cuda.mem_get_info()
    srv = pd.Server(int(0.6 * free), max_slots=slots, dt=DT, skin=SKIN, autotune=True)
    # tune every size bucket on throw-away systems first (untimed)
    for b in range(9, 19):
        n = int(min(2 ** b * 1.4, 262144))
        x, v, L = workloads.serving_system(n, 0.8, seed=77 + b)
        t = srv.submit(x, v, L, 2)
        srv.run_until_done([t])
        srv.release(t)
    # (1) capacity
    st0 = srv.stats()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tickets = [srv.submit(x, v, L, steps) for (x, v, L) in systems[:part]]
    srv.run_until_done(tickets)
    t_cap = time.perf_counter() - t0
    st1 = srv.stats()
    tm_cap = srv.timers()
    for t in tickets:
        srv.release(t)
    srv.completed(1 << 20)  # drain: the Poisson phases poll their own tickets
    cap_ps = (st1["particle_steps"] - st0["particle_steps"]) / t_cap
    cap_sys = part / t_cap

    # (2) Poisson arrivals at each load
    def poisson(load, subset, rseed):
        rng = np.random.default_rng(rseed)
        arr = np.cumsum(rng.exponential(1.0 / (load * cap_sys), size=len(subset)))
        pend = list(range(len(subset)))
        live, lat = {}, []
        t0 = time.perf_counter()
        s0 = srv.stats()
        while pend or live:
            now = time.perf_counter() - t0
            while pend and arr[pend[0]] <= now:
                k = pend.pop(0)
                x, v, L = subset[k]
                live[srv.submit(x, v, L, steps)] = arr[k]
            if not live:
                time.sleep(max(0.0, min(arr[pend[0]] - now, 0.01)))
                continue
            srv.tick()
            now = time.perf_counter() - t0
            for t in srv.completed():
                lat.append(now - live.pop(t))
                srv.release(t)
        t_run = time.perf_counter() - t0
        s1 = srv.stats()
        lat = np.array(lat)
        return {"offered_vs_capacity": load, "systems": len(subset),
                "systems_per_s": len(subset) / t_run, "systems_vs_capacity": len(subset) / t_run / cap_sys,
                "value": (s1["particle_steps"] - s0["particle_steps"]) / t_run, "unit": METRIC,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "p99_over_p50": float(np.percentile(lat, 99) / np.percentile(lat, 50))}
    phases = []
    for q, load in enumerate(loads):
        phases.append(poisson(load, systems[part * (q + 1): part * (q + 2)], seed + 1 + q))
    tuned = srv.tuned()
    tm_all = srv.timers()
    st_all = srv.stats()
    del srv
    for ph in phases:
        ph["vs_isolated"] = ph["value"] / iso
        ph["vs_capacity"] = ph["value"] / cap_ps
    ok = [ph for ph in phases if ph["p99_over_p50"] <= 3.0 and ph["vs_isolated"] >= 0.7]
    return {"workload": f"{n_systems} systems of the serving stream (N log-uniform in [512, 262144], density 0.8, "
                        f"r_cut 2.5, skin 0.3, {steps} velocity-Verlet steps, FP32 forces + Kahan, FP64 energies); "
                        f"{part} submitted at once (capacity), then {part} Poisson arrivals at each of "
                        f"{', '.join(str(l) for l in loads)} x capacity",
            "max_slots": slots, "mean_particles": float(sizes.mean()),
            "capacity": {"value": cap_ps, "unit": METRIC, "systems_per_s": cap_sys},
            "poisson": phases,
            "isolated_sequential": {"value": iso, "unit": METRIC, "systems": len(sub),
                                    "p50_ms": float(np.percentile(plain_lat, 50) * 1e3),
                                    "p99_ms": float(np.percentile(plain_lat, 99) * 1e3)},
            "target_p99_within_3x_p50_at_0.7_isolated": {
                "met": bool(ok), "highest_load_meeting_it": max((ph["offered_vs_capacity"] for ph in ok), default=None)},
            "note": "Poisson value = particle-steps of that phase / (last completion - first arrival), ramp-up and "
                    "drain included; vs_isolated = that value / the isolated sequential throughput; "
                    "systems_vs_capacity = systems completed per second / the capacity phase's systems per second",
            "tuned_shape_by_log2_size": {str(k): {"tile_width": v[0], "lanes_per_particle": v[1], "cta_threads": v[2]}
                                         for k, v in tuned.items()},
            "host_ms": {"capacity_phase": tm_cap, "total": tm_all, "ticks": st_all["ticks"],
                        "rebuilds": st_all["rebuilds"]}}


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (every rank gets it): the replicas' timed regions
    are bracketed by barriers, so the job takes as long as its slowest GPU."""
    import torch
    if dist is None:
        return ms
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, n_local, steps, ms_max):
    """Whole-job particle-steps/s of `world` replicas of n_local particles each."""
    return world * n_local * steps / (ms_max / 1000.0)


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--tiles", type=int, default=1, help="1: tiled shared-memory rows, 0: global-index rows")
    ap.add_argument("--tx", type=int, default=0, help="cells per tile along x (0: automatic)")
    ap.add_argument("--tpp", type=int, default=0, help="threads per particle in the pair kernel (0: 2)")
    ap.add_argument("--nside", type=int, default=N_SIDE,
                    help="lattice side (default 160: 4,096,000 particles; smaller sides are profiling cases)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="fp64: plain FP64 path; mixed: FP32 cell-local positions, Kahan sums, FP64 wrap/energies")
    ap.add_argument("--forms", default="all",
                    help="other workloads reported beside the main line: all, none, or a comma list of "
                         "precision,clustered,c1,sph,serving,symmetric,compaction")
    ap.add_argument("--clustered-steps", type=int, default=200, help="steps of the clustered precision form")
    ap.add_argument("--serve-systems", type=int, default=800, help="systems in the serving sample")
    a = ap.parse_args()
    TUNE.update(tiles=a.tiles, tx=a.tx, tpp=a.tpp, precision=a.precision)
    mixed = a.precision == "mixed"
    if a.warmup < 3:
        a.warmup = 3
    world, rank, local = dist_setup(a.gpus)

    if a.impl == "reference":
        if rank != 0:
            return 0
        val, threads, n_ref, rebuilds, t = reference_arm(a.steps, a.warmup)
        sample = (f"oracle FP64 restatement (reference CPU path not buildable here), {n_ref}-particle "
                  f"{'full system' if n_ref == N_SIDE ** 3 else 'sample of the same lattice (bounded run time)'}, "
                  f"{a.warmup} warm-up + {a.steps} timed velocity-Verlet steps incl. {rebuilds} list rebuilds, "
                  f"{threads} threads")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 * t / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(N_SIDE ** 3, world),
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return 0

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist

    from openfpm_pdata_b200 import pd
    pd.lib()
    x, v, L = make_workload(a.nside)
    n = x.shape[0]
    vd, md = build_system(pd, x, v, L)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    md.run(a.warmup, energies=False)  # includes the first list build
    md.set_timing(True)
    clocks = Clocks(local)
    barrier()
    clocks.start()
    l0 = pd.launch_count()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    E = md.run(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    launches = pd.launch_count() - l0
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    barrier()
    ms = max_over_ranks(ms, pg, "cuda")
    timers = md.timers()
    n_dom, mean_nn, max_nn = md.list_stats()
    builds = int(E[:, 3].sum())

    value = replica_value(world, n, a.steps, ms)
    # roofline of the dominant kernel (Verlet-list LJ force): algorithmic bytes per launch
    # = N * (position + 4 B row length + row entries + force): the FP64 tiled kernel stages
    # 24-byte (x, y) / z copies, 2-byte entries; the precision form 16-byte offsets, FP32 forces
    f_ms, f_cnt = timers["force"]
    f_avg_s = f_ms / max(f_cnt, 1) / 1000.0
    # tiled rows: 2-byte entries, the position record is staged once per tile (counted once);
    # mixed form: 16-byte FP32 offset records and FP32 forces.  The FP64 tiled kernel of
    # every step but a run's last also makes the next step's kick and drift in place of
    # storing the force: it reads the 32-byte position record, the velocity (24) and the
    # 32-byte build position and writes the record, the velocity and the 24-byte staging
    # copy (168 bytes, those of the separate kick-drift kernel it replaces); the launches
    # of the timed run average steps - 1 of those and one force store
    if mixed:
        alg_bytes = n * (16 + 4 + 2 * mean_nn + 12)
    elif a.tiles:
        drift_share = (a.steps - 1) / max(a.steps, 1)
        alg_bytes = n * (24 + 4 + 2 * mean_nn + drift_share * 168 + (1 - drift_share) * 24)
    else:
        alg_bytes = n * (32 + 4 + 4 * mean_nn + 24)
    peak, peak_kind = peaks()
    achieved = alg_bytes / f_avg_s / 1e9
    # secondary roofline of the FP64 pair kernel (its arithmetic, not HBM, is the
    # nearer ceiling): flops counted as executed -- distance 8 per row entry; inside
    # r_cut another 25 (sigma^2 / r^2 from the reciprocal seed by one series correction
    # 7, s6 2, force factor 4, three force FMAs 6, energy 4, virial 2); pairs inside
    # r_cut estimated from the density (4/3 pi r_cut^3 rho)
    rho = n / (L * L * L)
    in_cut = 4.18879 * R_CUT ** 3 * rho
    flops = n * (8 * mean_nn + 25 * in_cut)
    fma_peak = pd.measure_fma_rate(pd.PD_F32 if mixed else pd.PD_F64)
    kname = "k_vtile_lj_mixed" if mixed else ("k_vtile_lj_xyz" if a.tiles else "k_lj_verlet_f64")
    traffic = read_traffic(f"{kname}_lj4M.md") if a.nside == N_SIDE else None
    if traffic is not None and a.tiles and not mixed:
        # the drifting launches' traffic and the last launch's, averaged like alg_bytes
        plain = read_traffic(f"{kname}_lj4M.md", "traffic_bytes_per_launch_no_drift")
        if plain is not None:
            traffic = drift_share * traffic + (1 - drift_share) * plain

    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+kahan/f64-energy" if mixed else "f64", "data": "synthetic",
        "config": bench_config(n, world, a.nside, mixed),
        "verlet_list": {"rebuilds_in_timed_region": builds, "mean_row": round(mean_nn, 2), "max_row": max_nn,
                        "tile_cells": md.launch_shape()["tile_tx"]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "k_vtile_lj_mixed" if mixed else ("k_vtile_lj_xyz (FP64)" if a.tiles else
                                                                  "k_lj_verlet<double>"),
                     "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": f_avg_s * 1000.0,
                     "arith": {"unit": "TFLOP/s", "dtype": "f32" if mixed else "f64",
                               "achieved": flops / f_avg_s / 1e12, "flops_per_launch": flops,
                               "peak": fma_peak, "frac": flops / f_avg_s / 1e12 / fma_peak,
                               "peak_kind": "measured: vector FMA throughput kernel on this GPU "
                                            "(pd_measure_fma_rate, an FMA counts two flops)",
                               "nominal_peak": 75.0 if mixed else 37.0}},
        "phases_ms_per_step": {k: (tv[0] / max(tv[1], 1)) for k, tv in timers.items()},
        "gpu_launches": int(launches),
        "clocks": ck,
    }

    if not a.no_e2e:
        # end to end through the public C ABI: pinned host buffers in, K steps, energies and
        # final state out; wall clock around create + H2D + run + D2H (every rank its own
        # replica on its own GPU; the job's time is the slowest rank's)
        # host data in the ABI's layouts (positions [n][3], velocities [3][n]) in pinned memory
        xp = torch.from_numpy(x).pin_memory().numpy()
        vt = np.ascontiguousarray(v.T.astype(np.float32 if mixed else np.float64))
        vp = torch.from_numpy(vt).pin_memory().numpy()
        xo = torch.empty(x.shape, dtype=torch.float64).pin_memory().numpy()
        vo = torch.empty(vt.shape, dtype=torch.float32 if mixed else torch.float64).pin_memory().numpy()

        def e2e_pass(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            lo2, hi2, bc2 = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
            pt2 = pd.PD_F32 if mixed else pd.PD_F64
            vd2 = pd.VectorDist(n, lo2, hi2, bc2, R_CUT + SKIN, dtype=np.float64, props=[(pt2, 3), (pt2, 3)])
            vd2.hostToDevicePos(xp)
            vd2.hostToDevicePropSoA(0, vp)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            md2 = pd.MD(vd2, 0, 1, dt=DT, mass=MASS, skin=SKIN, eps=EPS, sigma=SIGMA, r_cut=R_CUT,
                        precision=pd.PREC_MIXED if mixed else pd.PREC_FP64)
            md2.set_tiles(bool(TUNE["tiles"]), TUNE["tx"], TUNE["tpp"])
            E2a = md2.run(1)  # the first list build and forces, and one step (returns after a synchronisation)
            t2 = time.perf_counter()
            E2 = np.concatenate([E2a, md2.run(steps - 1)])
            t3 = time.perf_counter()
            vd2.deviceToHostPos(with_ghost=False, out=xo)
            vd2.deviceToHostPropSoA(0, out=vo, with_ghost=False)
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            del md2, vd2  # their device blocks go back to the library's block cache
            assert np.isfinite(E2).all()
            return t4 - t0, {"create_and_h2d": (t1 - t0) * 1e3, "driver_first_build_and_step": (t2 - t1) * 1e3,
                             "remaining_steps": (t3 - t2) * 1e3, "d2h": (t4 - t3) * 1e3}

        # one untimed pass first, like the W warm-up steps of the device-timed run: a fresh
        # process's first device allocations of this size wait on the driver for a time
        # that depends on what ran on the GPU before it (measured 6 to 300 ms)
        w_s, w_ms = e2e_pass(max(a.warmup, 2))
        barrier()
        t_e2e, e2e_ms = e2e_pass(a.steps)
        t_e2e = max_over_ranks(t_e2e * 1000.0, pg, "cuda") / 1000.0
        out["e2e"] = {"value": world * n * a.steps / t_e2e, "unit": METRIC,
                      "h2d_bytes_per_step": world * (x.nbytes + v.nbytes) / a.steps,
                      "d2h_bytes_per_step": world * (32 + (xo.nbytes + vo.nbytes) / a.steps),
                      "includes": "create, H2D of positions+velocities from pinned memory, first list build, "
                                  "K steps, per-step energies and final state D2H into pinned memory; "
                                  "after one untimed warm-up pass of the same calls",
                      "phases_ms": e2e_ms, "warmup_pass_ms": w_ms}

    if rank == 0 and world == 1 and a.forms != "none":
        want = a.forms.split(",") if a.forms != "all" else ["precision", "clustered", "c1", "sph", "serving",
                                                                     "symmetric", "compaction"]
        forms = {}
        if "precision" in want and not mixed:
            forms["precision"] = form_precision(pd, torch, x, v, L, a.steps, a.warmup, value)
        if "clustered" in want:
            forms["clustered"] = form_clustered(pd, torch, steps=a.clustered_steps)
        if "c1" in want:
            forms["cell_list_every_step"] = form_cell_list_every_step(pd, torch)
        if "sph" in want:
            forms["sph"] = form_sph(pd, torch)
        if "serving" in want:
            forms["serving"] = form_serving(pd, torch, n_systems=a.serve_systems)
        if "symmetric" in want:
            forms["symmetric"] = form_symmetric(pd, torch, x, L)
        if "compaction" in want:
            forms["compaction"] = form_compaction(pd, torch)
        out["forms"] = forms

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        val, threads, k, rebuilds, t = cpu_reference(x, v, L, 20, budget_s=20.0)
        out["cpu_baseline"] = {"value": val, "unit": METRIC, "cores": threads, "kind": "port",
                               "sample": f"oracle FP64 on the full {n}-particle system, {k} steps incl. "
                                         f"{rebuilds} list rebuilds, {threads} OpenMP threads"}
    if rank == 0:
        print(json.dumps(out))
    del md, vd
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
