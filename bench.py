"""Benchmark of the multislice hot path on B200.

Workload (default, --config cbed): batched convergent-beam diffraction with
frozen phonons -- Si [001] 16x16x60 cells, 1024^2 sampling, 240 slices of
1.358 A, 300 kV, 20 mrad probe centred, 8 phonon configurations in one call.
One step = one full simulation (8 configurations x 240 slices = 1920
probe-slices).  Metric: probe*slice/s (higher is better).

  value : device-timed with CUDA events on the engine's stream; the pattern
          stays in HBM; atoms are handed over from host memory each step
          (3 MB) as part of the call.
  e2e   : the same public C-ABI call with host buffers, host->device atoms
          and device->host pattern inside every step, wall-clocked.

Multi-GPU (torchrun): each rank simulates its own 8 phonon configurations
(seed offset by rank) and the patterns are summed with one NCCL all-reduce
per step; weak scaling, time = max over ranks.

--impl reference times the reference's CPU implementation of the path, which
here is the FP64 C restatement under oracle/ (the reference itself has no CPU
path and does not build), on the host cores.
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

ALGO_BYTES_NOTE = ("per probe-slice: one FP32-complex read + write of the wave (16 N bytes) plus the FP32 potential "
                   "slice amortised over the waves sharing it (4 N / S)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cbed", choices=["cbed", "stem", "hrtem"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-vs-plain, adjoint and uneven-batch measurements")
    ap.add_argument("--pass-kernels", type=int, default=0, choices=[0, 1, 2, 3],
                    help="slice-pass kernel form: 0 classic per-slice launches, uneven batches in the slice engine "
                         "(default); 1 persistent pipelined; 2 persistent slice engine everywhere; 3 per-slice "
                         "launches everywhere")
    ap.add_argument("--potential-overlap", type=int, default=0, choices=[0, 1],
                    help="potentials: 0 all before the slice loop (default), 1 in chunks beside the slice passes")
    ap.add_argument("--tile-shape", type=int, default=-1, choices=[-1, 0, 1, 2, 3, 4, 5],
                    help="tile shape of the hot passes: -1 autotuned (default); bit 0 narrow rows, bit 1 narrow "
                         "columns, bit 2 one warp per column (1024-point columns)")
    ap.add_argument("--tune-cache", default="",
                    help="JSON file keeping the autotuner's choices (probe batch, tile shape) across runs")
    ap.add_argument("--cells-z", type=int, default=0, help="specimen thickness in unit cells (0: the workload's)")
    ap.add_argument("--nconf", type=int, default=0, help="phonon configurations (0: the workload's)")
    return ap.parse_args()


def workload(config: str, rank: int = 0, cells_z: int = 0, nconf: int = 0):
    from cudaem_b200 import workloads as wl
    if config == "cbed":
        from cudaem_b200 import replicas
        cz = cells_z or 60
        p, at = wl.cbed_si(cells=(16, 16, cz), nconf=nconf or 8)
        p = replicas.for_rank(p, rank)   # each rank its own phonon configurations
        units = p.pn_nconf * 4 * cz
        desc = {"workload": "CBED Si[001] 16x16x60 cells, 1024^2, 240 slices x 1.358 A, 300 kV, 20 mrad, "
                            "8 frozen-phonon configurations per call", "grid": 1024, "slices": 240,
                "phonon_configs": 8, "waves_per_potential": 1}
    elif config == "stem":
        p, at = wl.stem_sto(nconf=1, scan=(16, 16))
        units = 16 * 16 * 50
        desc = {"workload": "STEM ADF SrTiO3[001] 16x16x25 cells, 1024^2, 50 slices, 200 kV, 22 mrad, "
                            "16x16 probe positions of the 64x64 scan, one phonon configuration", "grid": 1024,
                "slices": 50, "probes": 256, "waves_per_potential": 256}
    else:
        p, at = wl.hrtem_sto()
        units = 40
        desc = {"workload": "HRTEM SrTiO3[001] 10x10x20 cells, 512^2, 40 slices, 200 kV plane wave + CTF",
                "grid": 512, "slices": 40, "waves_per_potential": 1}
    return p, at, units, desc


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(config: str, p_full, budget_s: float = 20.0):
    """The FP64 oracle on a bounded sample of the same workload, all host threads."""
    from cudaem_b200 import workloads as wl
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    if config == "cbed":
        p, at = wl.cbed_si(cells=(16, 16, 60), nconf=1)
        sample = ("1 of the 8 phonon configurations (240 slices) of the 1024^2 Si CBED workload, FP64 host "
                  "multislice; fp32 = the same with the wave, FFTs, transmission and propagator in FP32")
        t = time.perf_counter()
        orc.simulate_cbed(p, at)
        dt = time.perf_counter() - t
        units = 240
        t = time.perf_counter()
        orc.simulate_cbed_f32(p, at)
        dt32 = time.perf_counter() - t
        return {"value": units / dt, "unit": "probe*slice/s", "cores": threads, "kind": "port", "sample": sample,
                "seconds": dt, "fp32": {"value": units / dt32, "unit": "probe*slice/s", "seconds": dt32}}
    elif config == "stem":
        p, at = wl.stem_sto(nconf=1, scan=(2, 1))
        sample = "2 probes x 50 slices of the 1024^2 SrTiO3 STEM workload"
        t = time.perf_counter()
        orc.simulate_stem(p, at)
        dt = time.perf_counter() - t
        units = 2 * 50
    else:
        p, at = wl.hrtem_sto()
        sample = "the full 512^2 HRTEM workload (40 slices)"
        t = time.perf_counter()
        orc.simulate_tem(p, at)
        dt = time.perf_counter() - t
        units = 40
    return {"value": units / dt, "unit": "probe*slice/s", "cores": threads, "kind": "port", "sample": sample,
            "seconds": dt}


def extras(ctx, pass_kernels: int = 0):
    """The metric's other two legs, the uneven batch and the HRTEM image, each device-timed through
    the C ABI: batched STEM against the one-probe-per-launch path, the adjoint against a forward
    pass, the 64-instance uneven batch with its completion-latency percentiles and its roofline,
    and one 512^2 HRTEM image (a single wave).  The STEM batch is also timed in the persistent slice
    engine (pass-kernel form 2); the uneven batch runs in the engine by default and is also timed
    with per-slice launches (form 3)."""
    import ctypes as C

    import torch

    import cudaem_b200 as cb
    from cudaem_b200 import _abi as abi
    from cudaem_b200 import workloads as wl
    L = cb.lib()
    sim = cb.MulSimulator(ctx=ctx)
    out = {}

    # batched STEM vs plain (SrTiO3 16x16x25 cells, 1024^2, 50 slices, 22 mrad, ADF 60-200 mrad)
    def stem_rate(p, at, reps=2):
        sim.executionSTEM(p, at)
        best = None
        for _ in range(reps):
            sim.executionSTEM(p, at)
            r = p.scan_nx * p.scan_ny * 50 / (ctx.last_device_ms / 1e3)
            best = r if best is None else max(best, r)
        return best, ctx.last_probe_batch

    p, at = wl.stem_sto(nconf=1, scan=(16, 16))
    batched, B = stem_rate(p, at)
    q, _ = wl.stem_sto(nconf=1, scan=(4, 2), batch=1)
    ctx.set_graphs(False)
    b1, _ = stem_rate(q, at)
    ctx.set_graphs(True)
    g, _ = wl.stem_sto(nconf=1, scan=(2, 1))
    g.exec_mode = abi.MS_EXEC_PLAIN
    general, _ = stem_rate(g, at, reps=1)
    out["stem_batched_vs_plain"] = {
        "workload": "STEM ADF SrTiO3[001] 16x16x25 cells, 1024^2, 50 slices, 200 kV, 22 mrad, one phonon "
                    "configuration; batched: 16x16 probes in autotuned batches replayed from a CUDA graph; "
                    "plain: one probe per launch (8 probes), no graph; general scan: the reference's "
                    "run_STEM_general_simu form, potential regenerated per probe and slice (2 probes)",
        "unit": "probe*slice/s", "batched": batched, "autotuned_batch": B, "plain": b1, "ratio": batched / b1,
        "general_scan": general, "ratio_vs_general_scan": batched / general}
    ctx.set_pass_kernels(2)
    eng, _ = stem_rate(p, at)
    ctx.set_pass_kernels(pass_kernels)
    out["stem_batched_vs_plain"].update({"batched_engine": eng, "ratio_engine": eng / b1})

    # the batched STEM workload at its full size, one call: 64x64 probe positions x 10 phonon
    # configurations x 50 slices (2.05 M probe-slices), against the plain per-probe rate above
    p, at = wl.stem_sto()
    units_c3 = p.scan_nx * p.scan_ny * p.pn_nconf * 50
    sim.executionSTEM(p, at)
    full = units_c3 / (ctx.last_device_ms / 1e3)
    out["stem_batched_vs_plain"].update({
        "full_workload": "STEM ADF SrTiO3[001] 16x16x25 cells, 1024^2, 50 slices, 200 kV, 22 mrad, 64x64 probes on a "
                         "0.2 A step x 10 phonon configurations, one call (device time)",
        "full_batched": full, "full_autotuned_batch": ctx.last_probe_batch, "full_ms": ctx.last_device_ms,
        "full_ratio": full / b1})

    # adjoint vs forward (SrTiO3 10x10x40 cells, 512^2, 80 slices, 16 probes, checkpoints every 8)
    p, at, xy = wl.adjoint_sto(n_probe=16)
    V = ctx.projected_potential(p, at, conf=0)
    rng = np.random.default_rng(7)
    Vt = (V + 0.01 * np.abs(V) * rng.standard_normal(V.shape)).astype(np.float32)
    z0 = 0.5 * p.dz
    T = ctx.stem_forward_potential(p, Vt, z0, xy)
    Vd = torch.from_numpy(V).cuda()
    gVd = torch.empty_like(Vd)
    cp = p.c()
    xy = np.ascontiguousarray(xy, np.float64)
    T = np.ascontiguousarray(T, np.float32)
    I = np.empty((xy.shape[0], p.n_det), np.float32)
    dptr = xy.ctypes.data_as(C.POINTER(C.c_double))
    fptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    vptr = C.cast(C.c_void_p(Vd.data_ptr()), C.POINTER(C.c_float))
    gptr = C.cast(C.c_void_p(gVd.data_ptr()), C.POINTER(C.c_float))
    loss, g10, g30 = C.c_double(), C.c_double(), C.c_double()
    fw, bw = [], []
    for i in range(4):
        ctx.check(L.ms_stem_forward_potential(ctx.handle, C.byref(cp), vptr, V.shape[0], 1, z0, dptr, xy.shape[0],
                                              fptr(I)))
        fw.append(ctx.last_device_ms)
        ctx.check(L.ms_stem_backward(ctx.handle, C.byref(cp), vptr, V.shape[0], 1, z0, dptr, xy.shape[0], fptr(T),
                                     C.byref(loss), gptr, C.byref(g10), C.byref(g30)))
        bw.append(ctx.last_device_ms)
    f, b = min(fw[1:]), min(bw[1:])
    classes = ("row", "col", "probe", "row_store", "row_adj", "col_adj", "seed", "grad_probe")
    ctx.set_profiling(True)
    ctx.profile_reset()
    ctx.check(L.ms_stem_backward(ctx.handle, C.byref(cp), vptr, V.shape[0], 1, z0, dptr, xy.shape[0], fptr(T),
                                 C.byref(loss), gptr, C.byref(g10), C.byref(g30)))
    split = {k: round(ctx.profile(k)[1], 3) for k in classes}
    ctx.set_profiling(False)
    out["adjoint"] = {"workload": "differentiable STEM SrTiO3[001] 10x10x40 cells, 512^2, 80 slices, 200 kV, "
                                  "22 mrad, 16 probes, ADF loss, checkpoints every 8 slices",
                      "forward_ms": f, "backward_ms": b, "ratio": b / f, "backward_kernel_ms": split,
                      "note": "backward = loss, dL/dV, dL/dC10, dL/dC30 in one call (its own forward sweep included)"}

    # uneven batch: 64 CBED instances, 256^2..2048^2, 10-200 slices, 80-300 kV, 10-30 mrad
    jobs = wl.uneven_mix(64)
    peak, peak_kind = peaks()

    # the patterns stay in HBM (device outputs allocated once), as in the headline metric: host
    # outputs would add pageable copies whose cost depends on whether the host pages are mapped yet
    nj = len(jobs)
    ucp = (abi.ms_params * nj)()
    uca = (abi.ms_atoms * nj)()
    uco = (abi.ms_output * nj)()
    keep = []
    for i, (p_i, a_i) in enumerate(jobs):
        C.memmove(C.byref(ucp[i]), C.byref(p_i.c()), C.sizeof(abi.ms_params))
        uca[i] = a_i.c()
        keep.append(a_i)
        t = torch.empty((p_i.ny, p_i.nx), dtype=torch.float32, device="cuda")
        keep.append(t)
        uco[i].image_intensity = C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float))
        uco[i].on_device = 1
    ulat = np.zeros(nj, np.float64)

    def uneven(variant):
        ctx.set_pass_kernels(variant)
        best = None
        for rep in range(3):
            ctx.check(L.ms_simulate_many(ctx.handle, nj, ucp, uca, uco,
                                         ulat.ctypes.data_as(C.POINTER(C.c_double))))
            if rep > 0 and (best is None or ctx.last_device_ms < best[0]):
                best = (ctx.last_device_ms, ulat.copy())
        ctx.set_pass_kernels(pass_kernels)
        ms, lat = best
        ns = [uco[i].n_slices for i in range(nj)]
        units = sum(n_i * max(1, p.pn_nconf) for (p, _), n_i in zip(jobs, ns))
        # algorithmic bytes: per probe-slice 16 N (wave read + write) + 4 N (the instance's sigma V)
        algo = sum(20.0 * p.nx * p.ny * n_i * max(1, p.pn_nconf) for (p, _), n_i in zip(jobs, ns))
        gbs = algo / (ms / 1e3) / 1e9
        return {"unit": "probe*slice/s", "value": units / (ms / 1e3), "ms": ms, "probe_slices": units,
                "latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                               "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
                "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                             "peak_source": peak_kind, "algorithmic_bytes": algo,
                             "note": "whole call (specimens, potentials, slice passes, patterns) against the "
                                     "sum of every instance's 20 N bytes per probe-slice"}}

    out["uneven_batch"] = dict(workload="64 CBED instances drawn from seed 42: grids 256^2..2048^2, 10-200 slices "
                                        "of SrTiO3 or Si, 80-300 kV, 10-30 mrad, one phonon configuration each; "
                                        "every grid group in one persistent slice-engine launch (the default); "
                                        "latency = the device clock at which an instance's last wave was done",
                               **uneven(0))
    out["uneven_batch"]["per_slice_launches"] = uneven(3)
    out["uneven_batch"]["per_slice_launches"]["note"] = ("one row and one column launch per slice and grid group, "
                                                         "groups on their own streams; latency = each instance's "
                                                         "completion event")

    # HRTEM: one 512^2 plane wave, 40 slices, CTF image (a single wave: latency bound)
    p, at = wl.hrtem_sto()
    sim.executionTEM(p, at)
    t = []
    for _ in range(5):
        sim.executionTEM(p, at)
        t.append(ctx.last_device_ms)
    ms = min(t)
    ctx.set_profiling(True)
    ctx.profile_reset()
    sim.executionTEM(p, at)
    prof = {k: round(ctx.profile(k)[1], 4) for k in ("row", "col", "potential")}
    nl = {k: ctx.profile(k)[0] for k in ("row", "col")}
    ctx.set_profiling(False)
    host = time.perf_counter()
    for _ in range(5):
        sim.executionTEM(p, at)
    e2e_ms = (time.perf_counter() - host) * 1e3 / 5
    out["hrtem"] = {"workload": "HRTEM SrTiO3[001] 10x10x20 cells, 512^2, 40 slices, 200 kV plane wave, coherent "
                                "CTF image, one configuration", "unit": "probe*slice/s",
                    "value": 40 / (ms / 1e3), "ms": ms, "e2e": {"value": 40 / (e2e_ms / 1e3), "ms": e2e_ms},
                    "kernel_ms": prof, "launches": nl,
                    "slice_us": {k: 1e3 * prof[k] / max(1, nl[k]) for k in ("row", "col")}}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cudaem_b200 import workloads as wl  # noqa: F401
    from oracle import oracle as orc
    orc.build()
    _, _, _, desc = workload(args.config)
    times, units = [], 0
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(args.config, None)
        if i >= args.warmup:
            times.append(r["seconds"])
            units = r["value"] * r["seconds"]
    tot = sum(times)
    val = units * len(times) / tot
    line = {"impl": "reference", "metric": "probe*slice/s", "value": val, "unit": "probe*slice/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": desc,
            "cpu_baseline": {"value": val, "unit": "probe*slice/s", "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": val, "unit": "probe*slice/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# DRAM bytes (read + write) of one launch of a slice pass, from one ncu capture of the same launch
# (8 waves of 1024^2 in flight, caches not flushed, after the same command ran without ncu; the
# column step with wide tiles, the row step with narrow tiles, as the autotuner picks them):
# keyed by (workload, kernel class, grid, waves per launch)
DRAM_TRAFFIC = {
    ("cbed", "col", 1024, 8): 57.330944e6 + 39.807232e6,
    ("cbed", "row", 1024, 8): 106.883840e6 + 29.984768e6,
}


L2_BYTES = 126 * 1024 * 1024   # B200 L2


def run_ours(args):
    import ctypes as C

    import torch

    import cudaem_b200 as cb
    from cudaem_b200 import _abi as abi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    p, at, units, desc = workload(args.config, rank, args.cells_z, args.nconf)
    # the transmission store of every slice (8 bytes per pixel and slice, per configuration; one
    # configuration's store serves a STEM batch)
    store_bytes = 8 * p.nx * p.ny * (units if args.config != "stem" else 50)
    if args.cells_z or args.nconf:
        desc = dict(desc, workload=desc["workload"] + f" [reduced: cells_z={args.cells_z}, nconf={args.nconf}]")
    ctx = cb.Context(local)
    ctx.set_pass_kernels(args.pass_kernels)
    if args.tune_cache:
        ctx.set_tune_cache(args.tune_cache)
    ctx.set_tile_shape(args.tile_shape)
    ctx.set_potential_overlap(bool(args.potential_overlap))
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    L = cb.lib()
    N = p.nx * p.ny
    out_dev = torch.empty((p.ny, p.nx), dtype=torch.float32, device="cuda")
    co = abi.ms_output()
    cp, ca = p.c(), at.c()
    is_stem = args.config == "stem"
    if is_stem:
        out_dev = torch.empty((p.n_det, p.scan_ny, p.scan_nx), dtype=torch.float32, device="cuda")
        co.stem_intensity = C.cast(C.c_void_p(out_dev.data_ptr()), C.POINTER(C.c_float))
    else:
        co.image_intensity = C.cast(C.c_void_p(out_dev.data_ptr()), C.POINTER(C.c_float))
    co.on_device = 1
    fn = {"cbed": L.ms_simulate_cbed, "stem": L.ms_simulate_stem, "hrtem": L.ms_simulate_tem}[args.config]

    from cudaem_b200 import replicas

    def step(o):
        ctx.check(fn(ctx.handle, C.byref(cp), C.byref(ca), C.byref(o)))
        replicas.sum_patterns(out_dev, dist)

    for _ in range(args.warmup):
        step(co)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        # one more untimed step while the clock sampler starts (its start-up competes for the
        # host cores that issue the launches)
        step(co)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        if store_bytes >= L2_BYTES:
            ev0.record(stream)
            for _ in range(args.steps):
                step(co)
                launches += ctx.last_launch_count
            ev1.record(stream)
            torch.cuda.synchronize()
            t_ms = ev0.elapsed_time(ev1)
        else:
            # the slice store fits in L2: a 256 MiB write flushes L2 before every step, outside the
            # timed events (each step timed on its own, the times summed)
            flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
            t_ms = 0.0
            for _ in range(args.steps):
                flush.zero_()
                ev0.record(stream)
                step(co)
                ev1.record(stream)
                launches += ctx.last_launch_count
                torch.cuda.synchronize()
                t_ms += ev0.elapsed_time(ev1)
    ms = replicas.max_over_ranks(t_ms, device="cuda", dist=dist)
    value = units * world * args.steps / (ms / 1e3)

    # end to end: host atoms in, host pattern out, wall clock around the public call
    host_out = np.empty(tuple(out_dev.shape), np.float32)
    ch = abi.ms_output()
    if is_stem:
        ch.stem_intensity = host_out.ctypes.data_as(C.POINTER(C.c_float))
    else:
        ch.image_intensity = host_out.ctypes.data_as(C.POINTER(C.c_float))
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ctx.check(fn(ctx.handle, C.byref(cp), C.byref(ca), C.byref(ch)))
    e2e_s = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda", dist=dist)
    e2e = units * world * args.steps / e2e_s
    h2d = at.n * (4 * 6)
    d2h = host_out.nbytes

    # dominant kernel: per-launch device time from events around each launch (profiling run)
    ctx.set_profiling(True)
    ctx.profile_reset()
    step(co)
    torch.cuda.synchronize()
    prof = {k: ctx.profile(k) for k in ("row", "col", "potential", "probe", "engine")}
    prof = {k: v for k, v in prof.items() if v[0] > 0}
    ctx.set_profiling(False)
    dom = max(prof, key=lambda k: prof[k][1])
    n_l, tot_ms = prof[dom]
    waves = p.pn_nconf if args.config == "cbed" else (p.scan_nx * p.scan_ny if is_stem else 1)
    S_share = desc.get("waves_per_potential", 1)
    if dom in ("row", "col"):
        # one launch = one pass over the wave batch; algorithmic bytes per wave: read + write 8 N, plus
        # (row pass) the potential slice 4 N shared by S waves
        per_wave = 16 * N + (4 * N / S_share if dom == "row" else 0)
        algo = per_wave * waves
    elif dom == "engine":
        # one launch = every slice of the batch: a row and a column pass per wave and slice
        algo = units * (32 * N + 4 * N / S_share)
    else:
        algo = 4 * N * (p.pn_nconf if args.config == "cbed" else 1)
    avg_s = tot_ms / max(1, n_l) / 1e3
    achieved = algo / avg_s / 1e9
    peak, peak_kind = peaks()
    hbm_traffic = DRAM_TRAFFIC.get((args.config, dom, p.nx, waves))
    line = {"metric": "probe*slice/s", "value": value, "unit": "probe*slice/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32-complex (fp64 phases)", "data": "synthetic",
            "config": dict(desc, l2=(f"inputs larger than L2 (slice store {store_bytes / 1e9:.2f} GB)"
                                     if store_bytes >= L2_BYTES else
                                     f"slice store {store_bytes / 1e6:.0f} MB fits in L2: L2 flushed (256 MiB "
                                     f"write) before every step, outside the timed events"),
                           parallelism=f"phonon configurations per rank, {world} rank(s)"),
            "e2e": {"value": e2e, "unit": "probe*slice/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": hbm_traffic,
                         "launch_ms": avg_s * 1e3, "algorithmic_bytes_per_launch": algo,
                         "kernel_share": {k: v[1] for k, v in prof.items()}},
            "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_extras:
        line.update(extras(ctx, args.pass_kernels))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.config, p)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
