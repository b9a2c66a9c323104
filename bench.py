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


def read_traffic(kernel_file):
    """dram bytes per force launch (scaled to the full workload) from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", kernel_file)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
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
    a = ap.parse_args()
    TUNE.update(tiles=a.tiles, tx=a.tx, tpp=a.tpp, precision=a.precision)
    mixed = a.precision == "mixed"
    if a.warmup < 3:
        a.warmup = 3
    world, rank, local = dist_setup(a.gpus)

    if a.impl == "reference":
        if rank != 0:
            return 0
        x, v, L = make_workload()
        val, threads, k, rebuilds, t = cpu_reference(x, v, L, a.steps, budget_s=60.0)
        sample = (f"oracle FP64 restatement (reference CPU path not buildable here), full {x.shape[0]}-particle "
                  f"system, {k} velocity-Verlet steps incl. {rebuilds} list rebuilds, {threads} threads")
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": a.gpus, "steps": k,
            "warmup": 1, "ms_per_step": 1000.0 * t / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD},
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
    if pg is not None:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    timers = md.timers()
    n_dom, mean_nn, max_nn = md.list_stats()
    builds = int(E[:, 3].sum())

    value = world * n * a.steps / (ms / 1000.0)
    # roofline of the dominant kernel (Verlet-list LJ force): algorithmic bytes per launch
    # = N * (32 B position record + 4 B row length + 4 B * mean row + 24 B force)
    f_ms, f_cnt = timers["force"]
    f_avg_s = f_ms / max(f_cnt, 1) / 1000.0
    # tiled rows: 2-byte entries, the position record is staged once per tile (counted once);
    # mixed form: 16-byte FP32 offset records and FP32 forces
    if mixed:
        alg_bytes = n * (16 + 4 + 2 * mean_nn + 12)
    else:
        alg_bytes = n * (32 + 4 + (2 if a.tiles else 4) * mean_nn + 24)
    peak, peak_kind = peaks()
    achieved = alg_bytes / f_avg_s / 1e9
    kname = "k_vtile_lj_mixed" if mixed else ("k_vtile_lj_f64" if a.tiles else "k_lj_verlet_f64")
    traffic = read_traffic(f"{kname}_lj4M.md") if a.nside == N_SIDE else None

    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+kahan/f64-energy" if mixed else "f64", "data": "synthetic",
        "config": {"workload": workload_name(a.nside, mixed),
                   "particles": n, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (positions 131 MB + Verlet list ~1.1 GB per replica)",
                   "list_rebuilds_in_timed_region": builds, "mean_verlet_row": round(mean_nn, 2),
                   "max_verlet_row": max_nn},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "k_vtile_lj_mixed" if mixed else ("k_vtile_lj<double>" if a.tiles else
                                                                  "k_lj_verlet<double>"),
                     "peak_kind": peak_kind,
                     "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": f_avg_s * 1000.0},
        "phases_ms_per_step": {k: (tv[0] / max(tv[1], 1)) for k, tv in timers.items()},
        "gpu_launches": int(launches),
        "clocks": ck,
    }

    if rank == 0 and world == 1 and not a.no_e2e:
        # end to end through the public C ABI: pinned host buffers in, K steps, energies and
        # final state out; wall clock around create + H2D + run + D2H
        xp = torch.from_numpy(x).pin_memory().numpy()
        vp = torch.from_numpy(v).pin_memory().numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        vd2, md2 = build_system(pd, xp, vp, L)
        E2 = md2.run(a.steps)
        xo = vd2.deviceToHostPos(with_ghost=False)
        vo = vd2.deviceToHostProp(0, with_ghost=False)
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        del md2, vd2
        out["e2e"] = {"value": n * a.steps / t_e2e, "unit": METRIC,
                      "h2d_bytes_per_step": (x.nbytes + v.nbytes) / a.steps,
                      "d2h_bytes_per_step": 32 + (xo.nbytes + vo.nbytes) / a.steps,
                      "includes": "create, H2D of positions+velocities, first list build, K steps, "
                                  "per-step energies and final state D2H"}
        assert np.isfinite(E2).all()

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
