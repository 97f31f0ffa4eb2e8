#!/usr/bin/env python
"""Benchmark: one coarse Berger-Oliger step of grid transfers.

Workload (the 5-level order-5 hierarchy): 5 nested vertex-centred levels of
129^3 points, each split into 2x2x2 components, 25 FP64 grid functions with
3 timelevels, ghost width 3, buffer width 9; order-5 Lagrange boundary
prolongation with quadratic time interpolation across 3 timelevels,
injection restriction and ghost sync.  One step = every transfer of one
coarse step (the finest level takes 16 substeps).  Inputs are seeded
synthetic fields (4 Gaussians + 1e-6 noise).  Every step touches ~10 GB,
far more than the 126 MB L2, so no flush is needed between steps.

value        algorithmic GB/s of the batched form (one persistent kernel per
             phase, the step replayed as CUDA graphs), inputs resident in HBM
e2e          the same step through the public API with the grid data in
             pinned host memory: H2D of every array the step reads and D2H of
             every array it writes, inside the timed region (two device
             copies alternate so copy-in, kernels and copy-out overlap)
plain        the plain per-box form (one launch per box-pair), same step
roofline     the dominant kernel (the phase kind with the largest share of
             the step): its algorithmic bytes per launch / its CUDA-event time
cpu_baseline CarpetLib's own operators (compiled from the reference) on the
             host cores, a bounded sample of the same step
served       the served ensemble (64 hierarchies, Poisson request stream)
batched_uneven  256 uneven mixed box-pairs, autotuned + graph vs per box
moving_boxes the 8-level moving-box hierarchy: a coarse step and a regrid
             (host schedule + batched graph fill); --no-moving skips it

--impl reference: only the CPU reference arm (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "prolong/restrict/sync GB/s & % HBM roof; batched+served vs plain; p50/p99 ms"
WORKLOAD = "5 vc levels x 129^3 (2x2x2 comps), 25 GFs x 3 TLs, ghost 3, buffer 9, " \
           "order-5 Lagrange + 3-TL time interpolation, rf2 injection, ghost sync; " \
           "one coarse Berger-Oliger step"


# the kernel each phase kind of the step runs (batches are homogeneous)
PHASE_KERNELS = {
    ("prolong", 3): "k_tma_map<VC<5>, 3 TL quadratic> (prolongation + time interpolation)",
    ("prolong", 1): "k_tma_map<VC<5>, 1 TL> (prolongation)",
    ("restrict", 1): "k_stream_map<injection> (restriction)",
    ("sync", 1): "k_stream_map<copy, 1 TL> (ghost sync)",
}


# grid-function groups of the bench step (independent phase chains on
# separate streams, see carpet_b200.amr.BergerOliger)
GF_GROUPS = 2
# phases by which each further group starts after the first
GF_STAGGER = 0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=6)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="cgx", choices=["cgx", "reference"])
    p.add_argument("--ngf", type=int, default=25)
    p.add_argument("--npoints", type=int, default=129)
    p.add_argument("--levels", type=int, default=5)
    p.add_argument("--fp", default="exact", choices=["exact", "fma"],
                   help="exact: the reference's operation order with two roundings per "
                        "multiply-add (bit-exact); fma: fused multiply-adds")
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="host time of the CPU baseline leg of the GPU arm")
    p.add_argument("--ref-seconds", type=float, default=2.0,
                   help="host time per step of the reference arm (sets the grid functions per step)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--serve-seconds", type=float, default=1.0)
    p.add_argument("--serve-config", type=int, default=None,
                   help="tile configuration of the served prolongations (default SERVE_TILE_CONFIG)")
    p.add_argument("--no-tune", action="store_true", help="default tile configurations")
    p.add_argument("--tile-config", type=int, default=None,
                   help="pin every prolongation variant to this tile configuration instead of tuning")
    p.add_argument("--no-uneven", action="store_true", help="skip the batched uneven section")
    p.add_argument("--gf-groups", type=int, default=GF_GROUPS,
                   help="grid-function groups whose phase chains run on separate streams")
    p.add_argument("--gf-stagger", type=int, default=GF_STAGGER,
                   help="phases by which each further grid-function group starts after the first")
    p.add_argument("--chain", type=int, default=0, choices=[0, 1],
                   help="1: each coarse step as one chain launch (one persistent kernel with "
                        "per-grid-function dependency counters) instead of one launch per phase")
    p.add_argument("--max-ctas", type=int, nargs=2, default=[0, 0], metavar=("TMA", "STREAM"),
                   help="CTAs per SM of the TMA prolongation and the streaming kernels (0: all that "
                        "fit); below the limit, the grid-function groups' kernels share the SMs")
    p.add_argument("--no-moving", action="store_true",
                   help="skip the moving-box section (8 levels, ~51 GB on the device)")
    return p.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event (throttle) reasons, sampled every 10 ms by a
    thread through NVML while the timed region runs (nvidia-smi every 200 ms
    when NVML is not importable).  Reads only; changes no GPU setting."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, torch_device=0):
        self.dev, self.samples, self.smax, self.stop = torch_device, [], None, False
        self.proc = self.t = None

    def _handle(self, nv):
        import torch
        try:
            p = torch.cuda.get_device_properties(self.dev)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.dev)

    def _nvml_loop(self, nv, h):
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((float(sm), int(r)))
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.t.start()
        except Exception:
            self._smi()
        return self

    def _smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.sw_power_cap,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        bits = [0x4, 0x8, 0x20, 0x40]

        def read():
            for line in self.proc.stdout:
                f = [x.strip() for x in line.split(",")]
                try:
                    sm, self.smax = float(f[0]), float(f[1])
                except (ValueError, IndexError):
                    continue
                r = sum(b for b, v in zip(bits, f[2:6]) if v.lower() == "active")
                self.samples.append((sm, r))
        self.t = threading.Thread(target=read, daemon=True)
        self.t.start()

    def __exit__(self, *a):
        self.stop = True
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return None
        sm = sorted(s for s, _ in self.samples)
        reasons = set()
        for _, r in self.samples:
            for bit, name in self.REASONS.items():
                if r & bit:
                    reasons.add(name)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": self.smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- field
def gaussians(seed, L):
    """4 Gaussians: centres ~U(domain), widths ~U(0.05,0.3) L, amplitudes ~U(-1,1)"""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(rng.uniform(0, L, 3), rng.uniform(0.05, 0.3) * L, rng.uniform(-1, 1))
            for _ in range(4)]


def fill_storage(st, h, seed=1):
    import torch
    L = h.levels[0].box[3]
    gen = torch.Generator(device="cuda").manual_seed(seed)
    for l, lev in enumerate(h.levels):
        for tl in range(st.ntl):
            for g in range(st.ngf):
                gs = gaussians(seed * 1000 + g * 10 + tl, L)
                for c, comp in enumerate(lev.comps):
                    b = comp.exterior
                    t = st.data[l][tl][g][c].tensor
                    nz, ny, px = t.shape
                    x = b[0] + torch.arange(px, device="cuda", dtype=torch.float64) * b[6]
                    y = b[1] + torch.arange(ny, device="cuda", dtype=torch.float64) * b[7]
                    z = b[2] + torch.arange(nz, device="cuda", dtype=torch.float64) * b[8]
                    v = torch.zeros((nz, ny, px), dtype=torch.float64, device="cuda")
                    for (cen, w, a) in gs:
                        r2 = ((x - cen[0]) ** 2)[None, None, :] + ((y - cen[1]) ** 2)[None, :, None] \
                            + ((z - cen[2]) ** 2)[:, None, None]
                        v += a * torch.exp(-r2 / (w * w))
                    v += 1e-6 * torch.randn((nz, ny, px), generator=gen, device="cuda",
                                            dtype=torch.float64)
                    t.copy_(v)


# ----------------------------------------------------------------- CPU arm
def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference(h, ngf, seconds_per_step, steps, warmup):
    """CarpetLib's own operators on the host cores (oracle/_ref, compiled
    from the reference sources; OpenMP over every core with the reference's
    call_operator split): the WHOLE coarse Berger-Oliger step -- every phase
    of every level in the call order of Carpet/src/Evolve.cc:44-121, through
    data<T>::transfer_time with its per-call temporaries -- for as many grid
    functions as fit ``seconds_per_step`` (grid functions are independent,
    so the rate per grid function is the rate of the step).  Every build
    present is calibrated on one grid function; the fastest is timed over
    ``warmup`` + ``steps`` steps.  Returns a dict for the JSON line."""
    from carpet_b200 import bo
    from oracle.bo_step import RefStep, builds
    found = builds()
    if not found:
        return None
    L = len(h.levels)
    rates = {}
    cal = {}
    for name, path in found:
        rs = RefStep(h, 1, path=path)
        rot = [0] * L
        rs.run(bo.step_phases(L, 3, rot))  # warm: page in, build the call lists
        keys = bo.step_phases(L, 3, rot)
        t0 = time.perf_counter()
        nb = rs.run(keys)
        el = time.perf_counter() - t0
        rates[name] = round(nb / el / 1e9, 3)
        cal[name] = (path, el)
        del rs
    best = max(rates, key=rates.get)
    path, t1 = cal[best]
    ng = max(1, min(ngf, int(seconds_per_step / t1)))
    rs = RefStep(h, ng, path=path)
    rot = [0] * L
    for _ in range(max(1, warmup)):
        rs.run(bo.step_phases(L, 3, rot))
    total, el = 0, 0.0
    for _ in range(steps):
        keys = bo.step_phases(L, 3, rot)
        t0 = time.perf_counter()
        total += rs.run(keys)
        el += time.perf_counter() - t0
    v = total / el / 1e9
    return {"value": round(v, 3), "unit": "GB/s", "cores": host_cores(), "kind": "reference",
            "build": best, "builds_gbs": rates, "ms_per_step": round(el / steps * 1e3, 2),
            "sample": f"the whole coarse step (91 phases, 5 levels) for {ng} of the {ngf} grid "
                      f"functions per step, {steps} step(s) after {max(1, warmup)} warm-up; "
                      f"{total / 1e9:.2f} GB algorithmic in {el:.1f} s; fastest of "
                      f"{len(rates)} reference build(s)"}


# ----------------------------------------------------------------- served
# tile configuration of the served prolongations (the one the autotuner picks
# for the step): on the served ensemble configurations 0, 2 and 1 measured
# the same closed-loop rate (628-636 GB/s) and p50 0.42, 0.31 and 0.27 ms at
# 1e5 requests/s; configuration 4 was slowest in a closed-loop sweep
SERVE_TILE_CONFIG = 1


def served(seconds: float, peak_gbs: float, tile_config: int = SERVE_TILE_CONFIG):
    """The served ensemble: 64 independent 3-level hierarchies (coarse sizes
    U{24..64} per axis, 4 grid functions x 3 timelevels, 2 components per
    level, each with a regrid-fill operation), admitted against a 150 GB HBM
    budget.  Poisson request streams (sync/prolong/restrict 60/25/15) at 1e3,
    1e4 and 1e5 requests/s, each served continuously batched and through the
    plain per-box drop-in one request at a time; a stream with 5% regrid
    fills; and the closed-loop saturation point (every request submitted at
    once), with its algorithmic GB/s against the HBM roof."""
    import torch
    from carpet_b200.serve import (SERVE_BATCHED, SERVE_PLAIN, Ensemble, Server, ops_for,
                                   poisson_trace)
    out = {"workload": "64 hierarchies x 3 vc levels, coarse U{24..64}^3, 4 GFs x 3 TLs, "
                       "order-5 prolongation + 3-TL time interpolation; Poisson stream "
                       "sync/prolong/restrict 60/25/15", "budget_gb": 150,
           "tile_config": tile_config, "rates": []}
    warm = Server(mode=SERVE_BATCHED)
    ens = Ensemble(warm, nhier=64, size_range=(24, 64), seed=42, regrid=True)
    plain = Server(mode=SERVE_PLAIN)
    plain_ops = ens.define(plain)
    keys, arr = poisson_trace(ens, 1e4, 200, seed=1)   # warm-up: module load, attributes
    warm.replay(ops_for(ens.ops, keys), arr)
    warm.drain()
    plain.replay(ops_for(plain_ops, keys[:50]), arr[:50])
    plain.drain()
    plain.close()
    out["hierarchies"] = len(ens.members)
    out["hbm_gb"] = round(warm.report()["hbm_used"] / 1e9, 3)

    def run(mode, keys, arr):
        sv = Server(mode=mode)
        if mode == SERVE_BATCHED:
            sv.set_config(tile_config)
        op_ids = ens.define(sv)
        torch.cuda.synchronize()
        sv.replay(ops_for(op_ids, keys), arr)
        sv.drain()
        r = sv.report()
        sv.close()
        return {"requests": int(r["requests"]), "p50_ms": round(r["p50_ms"], 4),
                "p99_ms": round(r["p99_ms"], 4),
                "fine_points_per_s": round(r["points_per_s"], 1),
                "gbs": round(r["bytes_per_s"] / 1e9, 2),
                "launches": r["launches"], "mean_batch": round(r["mean_batch"], 2)}

    for rate in (1e3, 1e4, 1e5):
        n = int(min(rate * seconds, 20000))
        keys, arr = poisson_trace(ens, rate, n, seed=int(rate))
        row = {"rate_per_s": rate, "requests": n, "batched": run(SERVE_BATCHED, keys, arr)}
        # the plain drop-in falls behind at the highest rate: a bounded prefix
        m = n if rate <= 1e4 else min(n, 4000)
        row["plain"] = run(SERVE_PLAIN, keys[:m], arr[:m])
        out["rates"].append(row)
    keys, arr = poisson_trace(ens, 1e4, int(min(1e4 * seconds, 10000)), seed=77,
                              mix=(0.57, 0.24, 0.14, 0.05))
    out["with_regrid_fill"] = {"rate_per_s": 1e4, "mix": "sync/prolong/restrict/regrid-fill 57/24/14/5",
                               "batched": run(SERVE_BATCHED, keys, arr),
                               "plain": run(SERVE_PLAIN, keys, arr)}
    # closed loop: the whole stream submitted at once
    keys, _ = poisson_trace(ens, 1e5, 20000, seed=99)
    sat = {"requests": len(keys), "batched": run(SERVE_BATCHED, keys, [0.0] * len(keys)),
           "plain": run(SERVE_PLAIN, keys[:2000], [0.0] * 2000)}
    sat["batched"]["frac_hbm_roof"] = round(sat["batched"]["gbs"] / peak_gbs, 4)
    sat["batched_vs_plain"] = round(sat["batched"]["gbs"] / max(1e-9, sat["plain"]["gbs"]), 1)
    out["saturation"] = sat
    warm.close()
    return out


# ----------------------------------------------------------------- uneven
def uneven(steps: int, warmup: int, fp: str):
    """Batched uneven configuration: 256 box-pairs, fine extents U{16..96}
    per axis, operators 40/20/20/20 vc Lagrange o5 / vc ENO o3 / cc Lagrange
    o3 / cc averaging; autotuned tiles, one graph replay per step, against the
    plain per-box launches of the same descriptors."""
    import torch
    import carpet_b200 as cb
    from carpet_b200.uneven import uneven_batch, uneven_pairs, uneven_specs
    cb.set_fp_mode(fp == "fma")
    pairs = uneven_pairs(uneven_specs(seed=3, npairs=256, ext=(16, 96)), seed=4)
    b = uneven_batch(pairs)
    st = b.stats()
    tuned = b.autotune(reps=5)
    s = torch.cuda.Stream()
    g = cb.Graph()
    with g.capture(s):
        b.launch(s)

    def timed(fn, k):
        for _ in range(warmup):
            fn()
        s.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(k):
            fn()
        e.record(s)
        s.synchronize()
        return a.elapsed_time(e) / k

    ms = timed(lambda: g.launch(s), steps)
    batched = [p.dst.tensor.clone() for p in pairs]
    pms = timed(lambda: b.launch_per_box(s), max(1, steps // 2))
    same = all(torch.equal(x.view(torch.int64), p.dst.tensor.view(torch.int64))
               for x, p in zip(batched, pairs))
    b.check(s)
    return {"workload": "256 box-pairs, fine extents U{16..96}^3, 40% vc Lagrange o5, 20% vc ENO o3, "
                        "20% cc Lagrange o3, 20% cc averaging; autotuned, graph replay",
            "pairs": st["pairs"], "fine_points": st["points"], "bytes": st["bytes"],
            "ms": round(ms, 4), "gbs": round(st["bytes"] / (ms * 1e-3) / 1e9, 1),
            "fine_points_per_s": round(st["points"] / (ms * 1e-3), 1),
            "plain_ms": round(pms, 4), "plain_gbs": round(st["bytes"] / (pms * 1e-3) / 1e9, 1),
            "batched_vs_plain": round(pms / ms, 2), "identical_to_plain": bool(same),
            "tile_configs": sorted(set(tuned.values()))}


# ----------------------------------------------------------------- moving
def moving(ngf: int, fp: str, steps: int, peak_gbs: float):
    """Moving-box configuration: 8 vertex-centred levels (a 257^3 coarse level
    in 16 components; 7 refined levels of two 161^3 boxes, 8 components each,
    around two centres orbiting at 0.3 L, one revolution per 256 coarse
    steps), ngf grid functions x 3 timelevels.  Times one coarse
    Berger-Oliger step (order-5 prolongation with quadratic time
    interpolation, injection, sync; graph replay) and one regrid after 8
    coarse steps: the host schedule recompute (hierarchy, old-to-new pairs,
    descriptors) and the batched, graph-captured fill of every refined level
    and timelevel on the GPU."""
    import time
    import torch
    import carpet_b200 as cb
    from carpet_b200.amr import BergerOliger, Storage
    from carpet_b200.moving import MovingSpec, Regrid, build
    cb.set_fp_mode(fp == "fma")
    spec = MovingSpec()
    h0 = build(spec, 0)
    st = Storage(h0, ngf, 3)
    fill_storage(st, h0, seed=5)
    s = torch.cuda.Stream()
    # one coarse step (grid-function groups on streams, as the main step)
    bo = BergerOliger(h0, st, order_space=5, order_time=2, groups=min(GF_GROUPS, ngf))
    keys = bo.step_phases()
    tuned = bo.autotune(keys, reps=3)
    g = cb.Graph()
    with g.capture(s):
        bo.run(keys, s)
    g.launch(s)
    s.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(steps):
        g.launch(s)
    e.record(s)
    s.synchronize()
    step_ms = a.elapsed_time(e) / steps
    sst = bo.stats(keys)
    for b in bo.batches.values():
        b.check(s)
    del g
    # one regrid: host schedule, then the device fill
    t0 = time.perf_counter()
    h1 = build(spec, spec.regrid_every)
    tb = time.perf_counter()
    new = Storage(h1, ngf, 3, share=st, shared_levels=(0,))
    t1 = time.perf_counter()
    rg = Regrid(h0, h1, ngf, 3, lambda l, tl: st.data[l][bo.pool_index(bo.rot[l], tl)],
                lambda l, tl: (st.data[0][bo.pool_index(bo.rot[0], tl)] if l == 0 else new.data[l][tl]))
    rg.upload()
    t2 = time.perf_counter()
    rst = rg.stats()
    gr = rg.graph(s)
    gr.launch(s)
    s.synchronize()
    a.record(s)
    gr.launch(s)
    e.record(s)
    s.synchronize()
    fill_ms = a.elapsed_time(e)
    for b in rg.batches:
        b.check(s)
    out = {"workload": "8 vc levels: 257^3 coarse (16 comps) + 7 levels of two 161^3 boxes (16 comps) "
                       f"orbiting at 0.3 L; {ngf} GFs x 3 TLs, order-5 + quadratic time interpolation; "
                       "regrid after 8 coarse steps",
           "resident_gb": round(st.nbytes() / 1e9, 1),
           "step_ms": round(step_ms, 2), "step_gbs": round(sst["bytes"] / (step_ms * 1e-3) / 1e9, 1),
           "step_phases": len(keys), "step_kernels": sst["kernels"], "gf_groups": bo.groups,
           "regrid_host_ms": round((tb - t0 + t2 - t1) * 1e3, 1),
           "regrid_alloc_ms": round((t1 - tb) * 1e3, 1),
           "regrid_fill_ms": round(fill_ms, 3),
           "regrid_fill_gbs": round(rst["bytes"] / (fill_ms * 1e-3) / 1e9, 1),
           "step_frac_hbm_roof": round(sst["bytes"] / (step_ms * 1e-3) / 1e9 / peak_gbs, 4),
           "fill_frac_hbm_roof": round(rst["bytes"] / (fill_ms * 1e-3) / 1e9 / peak_gbs, 4),
           "regrid_pairs": rst["pairs"], "regrid_fine_points": rst["points"],
           "tile_configs": sorted({c for v in tuned.values() for c in v.values()})}
    del gr
    return out


# ----------------------------------------------------------------- main
def workload_config(args, bytes_step, points_step):
    """the workload, identical in both arms' JSON lines"""
    return {"workload": WORKLOAD, "levels": args.levels, "points_per_level": args.npoints,
            "components_per_level": 8, "ngf": args.ngf, "ntl": 3,
            "bytes_per_step": int(bytes_step), "fine_points_per_step": int(points_step),
            "l2": "inputs larger than L2 (~16 GB algorithmic per step)"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        # rank 0 alone; the other ranks exit without work.  Nothing here
        # loads libcgx.so: the schedule is the pure-Python one.
        if rank != 0:
            return
        from carpet_b200.hierarchy import nested
        h = nested(args.levels, args.npoints, ghost=3, buffer=9, order=5, native=False)
        from carpet_b200.bo import workload_totals
        bytes_step, points_step = workload_totals(h, args.ngf)
        ref = cpu_reference(h, args.ngf, args.ref_seconds, args.steps, args.warmup)
        if ref is None:
            print(json.dumps({"impl": "reference", "unavailable": "the reference operators are not "
                              "built (oracle/_ref): run make -C oracle ref where the sources are"}))
            return
        v = ref["value"]
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ref["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(args, bytes_step, points_step),
            "parallelism": f"host cores (OpenMP, {ref['cores']} threads)",
            "cpu_baseline": ref,
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return

    import torch
    from carpet_b200 import replicas
    if world > 1:
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        replicas.init("nccl", timeout_s=120)
    import carpet_b200 as cb
    from carpet_b200.amr import BergerOliger, Storage
    from carpet_b200.bo import fp64_ops, phase_pairs
    from carpet_b200.hierarchy import nested

    cb.set_fp_mode(args.fp == "fma")
    h = nested(args.levels, args.npoints, ghost=3, buffer=9, order=5)
    st = Storage(h, args.ngf, 3)
    fill_storage(st, h, seed=1 + rank)
    if args.chain:
        args.gf_groups, args.gf_stagger = 1, 0
    bo = BergerOliger(h, st, order_space=5, order_time=2, groups=args.gf_groups,
                      stagger=args.gf_stagger, chain=bool(args.chain), max_ctas=args.max_ctas)
    steps3 = [bo.step_phases() for _ in range(3)]  # the rotation repeats every 3 steps
    for keys in steps3:
        for k in keys:
            bo.group_batches(k)
    tuned, tuned_by_key = {}, {}
    if args.tile_config is not None:
        for keys in steps3:
            bo.set_config(keys, args.tile_config)
            for k in keys:
                tuned_by_key[k] = {v: args.tile_config for v in range(40)}
        tuned = {"all": {0: args.tile_config}}
    elif not args.no_tune and not args.chain:
        for keys in steps3:
            for k, v in bo.autotune(keys, reps=5).items():
                tuned_by_key[k] = v
                if v:
                    tuned[f"{k[0]}-ntl{k[3]}"] = v
    stats = [bo.stats(k) for k in steps3]
    bytes_step = sum(s["bytes"] for s in stats) / 3
    points_step = sum(s["points"] for s in stats) / 3
    # the library's count (from its descriptors) against the host count of
    # the schedule that the reference arm prints
    from carpet_b200.bo import workload_totals
    if (int(bytes_step), int(points_step)) != tuple(int(x) for x in workload_totals(h, args.ngf)):
        raise RuntimeError("algorithmic byte counts of the library and the schedule differ")
    kernels_step = 1 if args.chain else sum(s["kernels"] for s in stats) / 3
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    if args.chain:
        for keys in steps3:
            c = bo.chain(keys, stream)  # built and uploaded outside the captures
            if c.stats()["bytes"] != bytes_step:
                raise RuntimeError("the chain's algorithmic bytes differ from the step's")

    # capture the three step variants as graphs
    graphs = []
    for keys in steps3:
        g = cb.Graph()
        with g.capture(stream):
            bo.run(keys, stream)
        graphs.append(g)

    def barrier():
        replicas.barrier()
        torch.cuda.synchronize()

    # warm-up, then K timed steps
    for s in range(args.warmup):
        graphs[s % 3].launch(stream)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record(stream)
        for s in range(args.steps):
            graphs[(args.warmup + s) % 3].launch(stream)
        e1.record(stream)
        stream.synchronize()
    barrier()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1) / args.steps)
    for b in bo.batches.values():
        b.check(stream)
    for c in bo.chains.values():
        c.check(stream)
    value = replicas.job_throughput(bytes_step, world, ms) / 1e9
    fine_pts = replicas.job_throughput(points_step, world, ms)

    # per-launch timing of every phase (same stream, no graph): each phase
    # is a homogeneous batch, i.e. one kernel; the dominant kernel is the
    # phase kind with the largest share of the step.  Each phase is timed as
    # ONE launch over all grid functions (the step itself runs the groups'
    # smaller launches concurrently), so that each kernel's rate is measured
    # alone, with the tile configurations the step uses.
    keys = steps3[(args.warmup + args.steps) % 3]
    bo_ph = bo
    if args.gf_groups > 1:
        bo_ph = BergerOliger(h, st, order_space=5, order_time=2)
        for k in dict.fromkeys(keys):
            b = bo_ph.batch(k)
            for v, c in tuned_by_key.get(k, {}).items():
                b.set_config(c, v)
            b.upload(stream)
        stream.synchronize()
    launches = [(k, bo_ph.batch(k)) for k in keys]
    for k, b in launches:  # warm
        b.launch(stream)
    stream.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in launches]
    for (a, b_), (k, b) in zip(evs, launches):
        a.record(stream)
        b.launch(stream)
        b_.record(stream)
    stream.synchronize()
    phases = {}
    fp64_of = {}
    for (a, b_), (k, b) in zip(evs, launches):
        name = PHASE_KERNELS[(k[0], k[3])]
        e = phases.setdefault(name, {"launches": 0, "ms": 0.0, "bytes": 0})
        e["launches"] += 1
        e["ms"] += a.elapsed_time(b_)
        e["bytes"] += b.stats()["bytes"]
        if k not in fp64_of:
            pairs, _, _ = phase_pairs(h, k)
            fp64_of[k] = args.ngf * sum(fp64_ops(k[0], k[3], q.dstbox, q.srcbox, 5) for q in pairs)
        e["fp64_ops"] = e.get("fp64_ops", 0) + fp64_of[k]
    tot_ms = sum(e["ms"] for e in phases.values())
    # FP64 peak: 64 double-precision lanes per SM (B200) at the maximum SM clock
    sm_count = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    fp64_peak = 64 * sm_count * (clk.smax or 1965.0) * 1e6 / 1e12  # T ops/s
    for e in phases.values():
        e["gbs"] = round(e["bytes"] / (e["ms"] * 1e-3) / 1e9, 1)
        e["share"] = round(e["ms"] / tot_ms, 3)
        if e["fp64_ops"]:
            e["fp64_tops"] = round(e["fp64_ops"] / (e["ms"] * 1e-3) / 1e12, 3)
            e["fp64_frac"] = round(e["fp64_tops"] / fp64_peak, 4)
        e["ms"] = round(e["ms"], 3)
    dom = max(phases, key=lambda n: phases[n]["ms"])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = phases[dom]["gbs"]
    bytes_per_launch = phases[dom]["bytes"] / phases[dom]["launches"]

    # plain per-box form: one launch per box-pair, in call order on one
    # stream (the single-chain batches), same step
    plain = None
    if not args.no_plain:
        keys = steps3[0]
        bo_ph.run(keys, stream, per_box=True)  # warm
        stream.synchronize()
        a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        bo_ph.run(keys, stream, per_box=True)
        b_.record(stream)
        stream.synchronize()
        pms = a.elapsed_time(b_)
        plain = {"value": round(stats[0]["bytes"] / (pms * 1e-3) / 1e9, 3), "unit": "GB/s",
                 "ms_per_step": round(pms, 3), "launches_per_step": stats[0]["pairs"]}

    # end to end: grid data in pinned host memory; every step copies in all
    # it reads and copies out all it writes: every timelevel of every level,
    # since one coarse step rotates the finer levels through all their
    # timelevels (each substep writes ghost zones and boundary shells of its
    # current one).  Two device copies of the hierarchy alternate, so that a
    # step's copy-in overlaps the previous step's transfers and copy-out (the
    # two copy directions and the kernels run on three streams).
    e2e = None
    if not args.no_e2e:
        host = [[torch.empty_like(p, device="cpu").pin_memory() for p in lp] for lp in st.pools]
        for lp, hp in zip(st.pools, host):
            for p, q in zip(lp, hp):
                q.copy_(p)
        # one set of output buffers: the copy-out stream writes them in step order
        hout = [[torch.empty_like(p, device="cpu").pin_memory() for p in lp] for lp in st.pools]
        h2d = sum(p.numel() * 8 for lp in st.pools for p in lp)
        d2h = h2d
        stB = Storage(h, args.ngf, 3)
        for la, lb in zip(st.pools, stB.pools):
            for p, q in zip(la, lb):
                q.copy_(p)
        boB = BergerOliger(h, stB, order_space=5, order_time=2, groups=args.gf_groups,
                           stagger=args.gf_stagger, chain=bool(args.chain), max_ctas=args.max_ctas)
        stepsB = [boB.step_phases() for _ in range(3)]
        for keys in stepsB:
            for k in keys:
                for b in boB.group_batches(k):
                    for v, c in tuned_by_key.get(k, {}).items():
                        b.set_config(c, v)
                    b.upload()
        graphsB = []
        for keys in stepsB:
            if args.chain:
                boB.chain(keys, stream)  # built and uploaded outside the capture
            g = cb.Graph()
            with g.capture(stream):
                boB.run(keys, stream)
            graphsB.append(g)
        torch.cuda.synchronize()
        bufs = [(st, bo, graphs), (stB, boB, graphsB)]
        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        in_done = [torch.cuda.Event() for _ in range(2)]
        comp_done = [torch.cuda.Event() for _ in range(2)]
        out_done = [torch.cuda.Event() for _ in range(2)]
        used = [False, False]
        n_e2e = max(4, min(2 * args.steps, 8))

        def e2e_step(s):
            x = s % 2
            sto, _, gr = bufs[x]
            if used[x]:
                s_in.wait_event(out_done[x])  # the buffer's last step is copied out
            with torch.cuda.stream(s_in):
                for lp, hp in zip(sto.pools, host):
                    for p, q in zip(lp, hp):
                        p.copy_(q, non_blocking=True)
            in_done[x].record(s_in)
            stream.wait_event(in_done[x])
            gr[(s // 2) % 3].launch(stream)
            comp_done[x].record(stream)
            s_out.wait_event(comp_done[x])
            with torch.cuda.stream(s_out):
                for lp, hp in zip(sto.pools, hout):
                    for p, q in zip(lp, hp):
                        q.copy_(p, non_blocking=True)
            out_done[x].record(s_out)
            used[x] = True

        for s in range(2):
            e2e_step(s)
        torch.cuda.synchronize()
        a, b_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s_in)
        for s in range(n_e2e):
            e2e_step(s + 2)
        b_.record(s_out)
        torch.cuda.synchronize()
        ems = replicas.max_over_ranks(a.elapsed_time(b_) / n_e2e)
        e2e = {"value": round(replicas.job_throughput(bytes_step, world, ems) / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": round(ems, 3), "steps": n_e2e,
               "pipelining": "two device copies alternate; copy-in, kernels, copy-out on three streams"}
        for b in boB.batches.values():
            b.check(stream)
        for c in boB.chains.values():
            c.check(stream)
        del graphsB

    cpu = None
    if rank == 0 and not args.no_cpu:
        from carpet_b200.hierarchy import nested as nested_py
        cpu = cpu_reference(nested_py(args.levels, args.npoints, ghost=3, buffer=9, order=5,
                                      native=False),
                            args.ngf, args.cpu_seconds / 3, 2, 1)

    serve = None
    if rank == 0 and not args.no_serve:
        serve = served(args.serve_seconds, peak,
                       SERVE_TILE_CONFIG if args.serve_config is None else args.serve_config)

    batched_uneven = None
    if rank == 0 and not args.no_uneven:
        batched_uneven = uneven(max(args.steps, 3), args.warmup, args.fp)

    moving_boxes = None
    if rank == 0 and not args.no_moving:
        moving_boxes = moving(args.ngf, args.fp, 2, peak)

    # DRAM bytes per launch of the dominant kernel: the ratio of DRAM bytes
    # to algorithmic bytes that ncu measured on a smaller capture of the same
    # kernel (profiles/traffic.json), scaled to this launch
    traffic = None
    try:
        ratios = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        if dom in ratios:
            traffic = int(ratios[dom]["dram_per_algorithmic_byte"] * bytes_per_launch)
    except (OSError, ValueError, KeyError):
        traffic = None

    # parity statement: the exact mode is bit-exact with the reference's
    # operation order (tests compare bit patterns); the fused mode's error
    # per operator is the table tests/test_gpu_fma_error.py measured
    parity = {"fp_mode": args.fp,
              "vs_reference": "bit-exact with CarpetLib compiled without contraction "
                              "(tests/test_gpu_parity.py, tests/test_gpu_fullsize.py)"
              if args.fp == "exact" else
              "fused multiply-adds in the reference's order; |delta| per operator below"}
    try:
        tab = json.load(open(os.path.join(ROOT, "profiles", "fma_error_per_operator.json")))
        rows = tab["operators"]
        parity["fma_mode_error"] = {
            "source": tab["command"],
            "max_abs_over_eps_max_src": round(max(r["max_rel_eps_src"] for r in rows.values()), 3),
            "max_ulp": max(r["max_ulp"] for r in rows.values()),
            "per_operator": {k: [round(r["max_rel_eps_src"], 3), r["max_ulp"]] for k, r in rows.items()},
            "per_operator_key": "[max |fma - exact| / (eps max|source|), max per-point ulp]"}
    except (OSError, ValueError, KeyError):
        pass

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(args, bytes_step, points_step),
            "fp_mode": args.fp, "gf_groups": args.gf_groups, "gf_stagger": args.gf_stagger,
            "parallelism": "replicas" if world > 1 else "single GPU",
            "resident_gb": round(st.nbytes() / 1e9, 2),
            "tile_configs": {n: sorted(set(v.values())) for n, v in tuned.items()},
            "fine_points_per_s": round(fine_pts, 1),
            "pct_hbm_roof": round(100 * value / world / peak, 2),
            "pct_nominal_8tbs": round(100 * value / world / 8000.0, 2),
            "plain": plain,
            "batched_vs_plain": None if not plain else round(value / world / plain["value"], 2),
            "gpu_launches": int(round(kernels_step * args.steps)),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": dom, "algorithmic_bytes_per_launch": int(bytes_per_launch),
                         "launch": f"one launch over all {args.ngf} grid functions, timed alone",
                         "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks
                         else "fallback 6650 GB/s",
                         "fp64": None if not phases[dom].get("fp64_ops") else {
                             "achieved": phases[dom]["fp64_tops"], "peak": round(fp64_peak, 2),
                             "unit": "T ops/s", "frac": phases[dom]["fp64_frac"],
                             "ops_per_launch": int(phases[dom]["fp64_ops"] / phases[dom]["launches"]),
                             "ops": "multiplies and adds of the separable bit-exact evaluation",
                             "peak_source": "nominal: 64 FP64 lanes per SM x SMs x max SM clock"}},
            "phases": phases, "parity": parity,
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clk.summary(), "served": serve,
            "batched_uneven": batched_uneven, "moving_boxes": moving_boxes,
        }
        print(json.dumps(out))
    del graphs
    replicas.finish()


if __name__ == "__main__":
    main()
