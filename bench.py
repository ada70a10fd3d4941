"""Benchmark of the fault-stiffness build on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config h20]

Workload (default `h20`): the BP8 grid at h = 20 m, L_fault = 800 m,
L_normal = 400 m (81 x 81 x 21 nodes per side, 826,686 DOF), Omega_f = the
whole fault plane (l_f = L_fault), i.e. all 13,122 unit-slip columns of K.
One step = one build of those K columns by batched mixed-precision CG (FP32
stencil and vector updates, FP64 reliable updates, rtol 1e-10 on the FP64
true residual), traction extraction included; columns refill CG slots as
others finish. Inputs are unit slips (synthetic by definition; no dataset is
involved). `--config h50` runs the h = 50 m grid (2,178 columns).

Prints one JSON line (rank 0). `value` = K columns/s with K written to
device memory; `e2e` = the same through the public host API (`fault_stiffness`
into a host array, every step). `serving` = per-request latency of a short
seeded Poisson mix of column requests over the four BP8 grids answered by the
continuous-batching server. Under torchrun (N > 1) each rank builds a
contiguous shard of the columns on its own GPU (no collective on the data
path); the step time is the max over ranks.
"""
import argparse
import ctypes as C
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

METRIC = "K columns/s at K rel err <=1e-8 (batched mixed-precision CG vs plain FP64 CG); solve p99 ms"
CONFIGS = {
    # name: dz, L_fault, L_normal, l_f
    "h100": (100.0, 800.0, 800.0, 800.0),   # 17x17x9 (the reference's 17x17x5 case needs >= 9 normal nodes)
    "h50": (50.0, 800.0, 400.0, 800.0),     # 33x33x9, 2,178 columns
    "h20": (20.0, 800.0, 400.0, 800.0),     # 81x81x21, 13,122 columns
    "h25": (25.0, 1600.0, 800.0, 1600.0),   # 129x129x33, 3.3 M DOF: 2,048 seeded columns + the 10 Toeplitz solves
}
# Per-config sample sizes: (K-error check columns, plain single-RHS columns,
# batched-FP64 columns, CPU-port columns); None = all columns.
SAMPLES = {
    "h100": (None, 24, None, 256),
    "h50": (None, 24, None, 256),
    "h20": (256, 4, 1024, 16),
    "h25": (64, 2, 256, 16),
}


def workload_columns(cfg, nf):
    """The K columns one step builds: all 2nf, or at h = 25 m the 2,048
    columns drawn without replacement by default_rng(4)."""
    if cfg == "h25":
        return np.sort(np.random.default_rng(4).choice(2 * nf, size=2048, replace=False)).astype(np.int32)
    return np.arange(2 * nf, dtype=np.int32)
MU = 32.04e9
NU = 0.25


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="h20")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=48, help="requests of the serving mix (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=100.0, help="Poisson arrival rate of the serving mix (req/s)")
    ap.add_argument("--columns", type=int, default=0,
                    help="build only the first N columns of the workload (profiler captures of a smaller case; "
                         "0: all)")
    return ap.parse_args()


def workload_name(cfg):
    dz, Lf, Ln, lf = CONFIGS[cfg]
    n1 = int(round(Ln / dz)) + 1
    n23 = int(round(2 * Lf / dz)) + 1
    nf = (int(round(2 * lf / dz)) + 1) ** 2
    ncols = 2048 if cfg == "h25" else 2 * nf
    what = f"{ncols} seeded unit-slip columns of {2 * nf}" if ncols != 2 * nf else f"{2 * nf} unit-slip columns"
    return (f"bp8 fault stiffness h={dz:g}m L_fault={Lf:g} L_normal={Ln:g} l_f={lf:g}: "
            f"{n23}x{n23}x{n1} nodes/side ({6 * n1 * n23 * n23} DOF), {what}"), n1, n23, nf


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_port_sample(cfg, ncols_sample, seed=0, threads=0):
    """The oracle's C restatement of the reference column loop (assembled CSR
    A, FP64 CG, Krylov rule), all host threads, on a seeded column sample."""
    from oracle.fault import FaultElasticity as OFE, bp8_grids, lame_lambda
    from oracle.cref import CRefStiffness, max_threads
    dz, Lf, Ln, lf = CONFIGS[cfg]
    gm, gp = bp8_grids(dz, Lf, Ln)
    ofe = OFE(gm, gp, lame_lambda(MU, NU), MU, lf)
    ref = CRefStiffness(ofe)
    rng = np.random.default_rng(seed)
    cols = np.sort(rng.choice(2 * ofe.nf, size=min(ncols_sample, 2 * ofe.nf), replace=False))
    nt = threads if threads > 0 else max_threads()
    return ofe, ref, cols, nt


def apply_kernel_name(variant, n1, tile_rows, threads):
    """The FP32 CG apply kernel a launch variant runs: variants 9 and 10 are
    the ring march on the lines it is built for (a CTA of 2 x roundup32(t2 n1)
    + roundup32(2 t2) threads), every other variant the plane march."""
    r32 = lambda x: (x + 31) // 32 * 32
    if variant >= 9 and threads == 2 * r32(tile_rows * n1) + r32(2 * tile_rows):
        return f"ring_march_kernel<n1={n1},t2={tile_rows}>"
    return "plane_march_kernel<float,MODE_A>"


def cpu_model():
    """The host CPU's model name (first processor of /proc/cpuinfo)."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


SERVE_GRIDS = {  # h: (dz, L_fault, L_normal, weight); Omega_f = the whole fault plane
    100: (100.0, 800.0, 800.0, 0.4),
    50: (50.0, 800.0, 400.0, 0.3),
    25: (25.0, 1600.0, 800.0, 0.2),
    20: (20.0, 800.0, 400.0, 0.1),
}


def serving_leg(eqd, device, nreq, rate, check=4, seed=5):
    """The serving mix (Poisson arrivals at `rate` req/s; grid h in {100, 50,
    25, 20} m with weights .4/.3/.2/.1; floor(exp(U(0, ln 512))) + 1 seeded
    unit-slip columns per request; HBM budget 150 GB) through the
    continuous-batching server. Latency = submit -> last K column delivered
    to the request's host buffer, per request."""
    from eqd_b200.serving import run_mix
    lam = eqd.lame_lambda(MU, NU)
    srv = eqd.Server(hbm_budget_bytes=int(150e9))
    fes, weights = [], []
    for h, (dz, Lf, Ln, w) in SERVE_GRIDS.items():
        fe = eqd.FaultElasticity(eqd.bp8_grids(dz, Lf, Ln), lam, MU, Lf, device=device)
        srv.add(fe, slots=512)
        fe.h = h
        fes.append(fe)
        weights.append(w)
    for fe in fes:  # first graph launches and tuning of every grid, untimed
        srv.submit(fe, [fe.nf // 2 + fe.n2f // 2]).wait(900)
    rng = np.random.default_rng(seed)
    reqs, wall = run_mix(srv, fes, weights, rate, nreq, rng)
    infos = [r.info() for r in reqs]
    lat = np.array([i["latency"] for i in infos]) * 1e3
    ncols = int(sum(i["ncols"] for i in infos))
    span = max(i["t_done"] for i in infos) - min(i["t_submit"] for i in infos)
    by_grid = {}
    for r, i in zip(reqs, infos):
        by_grid.setdefault(r.fe.h, []).append(i["latency"] * 1e3)
    srv.close()
    errs = []
    chk = {}
    for r in reqs[:check]:
        if r.fe.h not in chk:
            dz, Lf, Ln, _ = SERVE_GRIDS[r.fe.h]
            chk[r.fe.h] = eqd.FaultElasticity(eqd.bp8_grids(dz, Lf, Ln), lam, MU, Lf, device=device,
                                              precision="fp64", rtol=1e-12)
        K64 = eqd.stiffness_columns(chk[r.fe.h], r.cols)[0]
        errs.append(float(np.linalg.norm(r._out - K64) / np.linalg.norm(K64)))
    for fe in chk.values():
        fe.close()
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "columns_per_s": ncols / span, "requests": len(reqs), "columns": ncols,
            "rate_req_s": rate, "unconverged": int(sum(i["unconverged"] for i in infos)),
            "p50_ms_by_grid_h": {str(h): float(np.percentile(v, 50)) for h, v in sorted(by_grid.items())},
            "p99_ms_by_grid_h": {str(h): float(np.percentile(v, 99)) for h, v in sorted(by_grid.items())},
            "k_rel_err_max": max(errs) if errs else None, "k_rel_err_requests_checked": len(errs),
            "what": "per-request latency, submit -> last K column in the request's host buffer"}


def run_reference(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    wl, n1, n23, nf = workload_name(args.config)
    ofe, ref, cols, nt = cpu_port_sample(args.config, 64 if args.config in ("h100", "h50") else 16)
    for _ in range(args.warmup):
        ref.columns(cols[: max(1, len(cols) // 8)], nthreads=nt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, it, ok = ref.columns(cols, nthreads=nt)
    dt = (time.perf_counter() - t0) / args.steps
    v = len(cols) / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "columns/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (unit slips)",
        "config": {"workload": wl, "sample_columns": int(len(cols)), "mean_iterations": float(np.mean(it))},
        "cpu_baseline": {"value": v, "unit": "columns/s", "cores": nt, "cpu_model": cpu_model(), "kind": "port",
                         "sample": f"{len(cols)} seeded columns of the workload per step (C restatement of the "
                                   "reference column loop, assembled CSR A, FP64 Krylov-rule CG, OpenMP over columns)"},
        "e2e": {"value": v, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    world, rank, local = dist_init(args)
    from __graft_entry__ import import_package
    eqd = import_package()
    import torch
    from eqd_b200.sharding import shard_range

    dz, Lf, Ln, lf = CONFIGS[args.config]
    wl, n1, n23, nf = workload_name(args.config)
    n_err, n_plain, n_b64, n_cpu = SAMPLES[args.config]
    all_cols = workload_columns(args.config, nf)
    if args.columns > 0:
        all_cols = all_cols[: args.columns]
    ncols = len(all_cols)
    lo, hi = shard_range(ncols, rank, world)
    cols = all_cols[lo:hi]
    g = eqd.bp8_grids(dz, Lf, Ln)
    lam = eqd.lame_lambda(MU, NU)
    fe = eqd.FaultElasticity(g, lam, MU, lf, device=local, precision="mixed")
    lib = eqd._abi.lib()
    opts = fe.rs.opts()
    opts.itmax = 20000  # safety cap (a converging column needs a few hundred)
    if args.config in ("h20", "h25"):
        # Slot pool within 100 GiB (h = 20 m: ~5,000 slots, h = 25 m: ~1,300):
        # columns refill slots as others finish, and the rest of HBM stays free
        # for the comparisons below.
        opts.hbm_budget_bytes = 100 << 30
    kdev = torch.empty((len(cols), 2 * nf), dtype=torch.float64, device=f"cuda:{local}")

    def device_step():
        st = eqd._abi.Stats()
        eqd._abi.check(lib.eqd_stiffness_columns_device(
            fe.handle, eqd._abi.ptr(cols), C.c_int32(len(cols)), C.byref(opts),
            C.c_void_p(kdev.data_ptr()), None, None, C.byref(st)))
        return st

    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()
    barrier(world)
    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    dev_s, launches, step_ms, iters = [], 0, [], 0
    # Profiler brackets: under `ncu --profile-from-start off` only the timed
    # steps' launches are captured (no-ops otherwise).
    torch.cuda.profiler.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st = device_step()
        dev_s.append(st.device_seconds)
        step_ms.append(st.device_seconds * 1e3)
        launches += st.kernel_launches
        iters += st.iterations
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    torch.cuda.profiler.stop()
    clocks = clk.stop()
    barrier(world)
    dev_total = barrier_max(world, float(sum(dev_s)))
    ms_per_step = dev_total / args.steps * 1e3
    value = ncols / (dev_total / args.steps)
    mean_it = iters / (args.steps * len(cols))

    # End to end through the public API: host K every step.
    e2e_steps = max(1, min(args.steps, 3 if ncols * nf < 4e7 else 1))
    Kh = eqd.stiffness_columns(fe, cols)[0]
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        Kh, it_h, st_h = eqd.stiffness_columns(fe, cols)
    e2e_dt = barrier_max(world, (time.perf_counter() - t0) / e2e_steps)
    e2e = {"value": ncols / e2e_dt, "unit": "columns/s", "h2d_bytes_per_step": int(len(cols) * 4 * 3),
           "d2h_bytes_per_step": int(len(cols) * 2 * nf * 8 + len(cols) * 5)}

    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    Kmix = kdev.cpu().numpy().T

    # Autotuner evidence: every FP32 launch variant timed on the batch.
    sel = C.c_int32()
    nv = C.c_int32()
    tms = (C.c_double * 16)()
    trows = (C.c_int32 * 16)()
    tthr = (C.c_int32 * 16)()
    # ncols = 0: report the choice the timed steps ran with (tuned on first use), no re-tuning.
    eqd._abi.check(lib.eqd_autotune(fe.handle, C.c_int32(0), C.byref(sel), tms, trows, tthr, C.byref(nv)))
    autotune = {"selected": sel.value,
                "variants": [{"tile_rows": trows[i], "threads": tthr[i], "ms_per_cg_iteration": tms[i]}
                             for i in range(nv.value)]}
    kernel = apply_kernel_name(sel.value, n1, trows[sel.value], tthr[sel.value])
    # Chunk-width tuner (after the timed steps, which ran at the budget's width).
    widths = [w for w in (32, 64, 128, 256, 512, 1024, 2048, 4096) if w <= len(cols)]
    cbest, ctable = eqd.tune_chunk(fe, widths)
    chunk_tuning = {"best": cbest, "ms_per_column_iteration": {str(w): m for w, m in ctable},
                    "timed_steps_width": "HBM budget (100 GiB at h = 20 m and 25 m, else free memory)"}

    # Roofline of the dominant kernel: FP32 stencil apply over the batch.
    ms = C.c_double()
    by = C.c_double()
    napply = min(len(cols), 2178 if args.config in ("h100", "h50") else 512)
    eqd._abi.check(lib.eqd_profile_apply(fe.handle, C.c_int32(napply), C.c_int32(eqd._abi.EQD_PREC_MIXED),
                                         C.c_int32(3), C.c_int32(10), C.byref(ms), C.byref(by)))
    achieved = by.value / (ms.value * 1e-3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tp = os.path.join(ROOT, "profiles", "apply_traffic.json")
    if os.path.exists(tp):
        t = json.load(open(tp)).get(args.config, {}).get(kernel.split("<")[0])
        if t:
            traffic = t["dram_bytes_per_launch_per_column"] * napply

    # Time-loop GEMV on the resident K (full square K only).
    gemv = None
    if ncols == 2 * nf and 2 * nf <= 524288:  # static-scratch GEMV limit: n * nvec <= 524,288
        n = 2 * nf
        nvec = 1
        s = torch.from_numpy(np.random.default_rng(0).standard_normal(n)).to(kdev.device)
        y = torch.empty_like(s)
        stream = torch.cuda.current_stream(kdev.device)
        Kd = kdev  # row c of kdev = column c of K: column-major K
        for _ in range(3):
            eqd._abi.check(lib.eqd_kmat_gemv_static(C.c_int32(local), C.c_int32(n), C.c_void_p(Kd.data_ptr()),
                                                    C.c_void_p(s.data_ptr()), C.c_void_p(y.data_ptr()),
                                                    C.c_int32(nvec), C.c_void_p(stream.cuda_stream)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reps = 20
        for _ in range(reps):
            lib.eqd_kmat_gemv_static(C.c_int32(local), C.c_int32(n), C.c_void_p(Kd.data_ptr()),
                                     C.c_void_p(s.data_ptr()), C.c_void_p(y.data_ptr()), C.c_int32(nvec),
                                     C.c_void_p(stream.cuda_stream))
        e1.record(stream)
        torch.cuda.synchronize()
        gms = e0.elapsed_time(e1) / reps
        yref = Kmix @ s.cpu().numpy()
        gemv = {"n": n, "ms": gms, "GB_s": 8.0 * n * n / (gms * 1e-3) / 1e9,
                "rel_err_vs_host": float(np.linalg.norm(y.cpu().numpy() - yref) / np.linalg.norm(yref)),
                "slip": "N(0, 1 m^2), default_rng(0)"}

    # Batched K S for 64 slip vectors (Runge-Kutta stages / ensembles): the
    # blocked path reads K once per 64 vectors. Timed through the host API
    # (slips in, tractions out, every call).
    gemm = None
    if ncols == 2 * nf:
        n = 2 * nf
        nv = 64
        Sm = np.asfortranarray(np.random.default_rng(2).standard_normal((n, nv)))  # column-major, as a Julia caller holds it
        KM = eqd.KMatrix(Kmix)
        KM.gemv(Sm)
        reps = 5
        t0 = time.perf_counter()
        for _ in range(reps):
            Ym = KM.gemv(Sm)
        gdt = (time.perf_counter() - t0) / reps
        # The same product on device-resident slips (eqd_kmat_gemv_device):
        # the blocked kernel and its slice reduction, timed by CUDA events.
        sd = torch.from_numpy(np.ascontiguousarray(Sm.T)).to(f"cuda:{local}")
        yd = torch.empty_like(sd)
        stream = torch.cuda.current_stream()
        KM.gemv_device(sd, yd, stream=stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dreps = 10
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(dreps):
            KM.gemv_device(sd, yd, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        dms = e0.elapsed_time(e1) / dreps
        Ydev = yd.cpu().numpy().T
        KM.close()
        Yref = Kmix @ Sm
        props = torch.cuda.get_device_properties(local)
        sm_max = (clocks or {}).get("sm_max_mhz") or 1965.0
        fp64_peak = props.multi_processor_count * 128 * sm_max * 1e6 / 1e12
        dtf = 2.0 * n * n * nv / (dms * 1e-3) / 1e12
        gemm = {"n": n, "nvec": nv, "ms": gdt * 1e3, "GFLOP_s": 2.0 * n * n * nv / gdt / 1e9,
                "K_GB_s": 8.0 * n * n / gdt / 1e9,
                "rel_err_vs_host": float(np.linalg.norm(Ym - Yref) / np.linalg.norm(Yref)),
                "what": "eqd_kmat_gemv with 64 vectors through the host API (copies of S and Y included)",
                "device": {"ms": dms, "TFLOP_s": dtf, "peak_TFLOP_s": fp64_peak, "frac": dtf / fp64_peak,
                           "peak_kind": "nominal FP64 (SMs x 128 flop/clk x max SM clock)",
                           "same_bits_as_host_api": bool(np.array_equal(Ydev, Ym)),
                           "what": "eqd_kmat_gemv_device on resident slips, CUDA events, 10 calls"}}

    # The Toeplitz mode's 10 source solves (src/FaultResponse.jl:339-393:
    # the centre node, then the four corners, each with s2 and s3) on the
    # large grid, batched, checked against FP64 single-RHS CG.
    toeplitz = None
    if args.config == "h25":
        n2f = n3f = int(round(np.sqrt(nf)))
        nodes = [((n3f + 1) // 2 - 1) * n2f + (n2f + 1) // 2 - 1, 0, n2f - 1, (n3f - 1) * n2f, nf - 1]
        tcols = np.array([k + j * nf for k in nodes for j in (0, 1)], dtype=np.int32)
        Kt, itt, _ = eqd.stiffness_columns(fe, tcols)
        t0 = time.perf_counter()
        Kt, itt, _ = eqd.stiffness_columns(fe, tcols)
        tdt = time.perf_counter() - t0
        p1 = eqd.FaultElasticity(g, lam, MU, lf, device=local, precision="fp64", chunk=1, rtol=1e-12)
        Kt64 = np.column_stack([eqd.stiffness_columns(p1, [c])[0][:, 0] for c in tcols])
        p1.close()
        toeplitz = {"solves": int(len(tcols)), "wall_s": tdt, "mean_iterations": float(np.mean(itt)),
                    "k_rel_err_vs_fp64_single_rhs": float(np.linalg.norm(Kt - Kt64) / np.linalg.norm(Kt64))}

    fe.close()  # release the batch's slot pool before the FP64 comparisons

    # Accuracy of this K against a tight FP64 solve of the same columns (GPU
    # plain FP64 CG, rtol 1e-12), on all columns or a seeded sample.
    rng = np.random.default_rng(1)
    if n_err is None or n_err >= len(cols):
        pick = np.arange(len(cols))
    else:
        pick = np.sort(rng.choice(len(cols), size=n_err, replace=False))
    fe64 = eqd.FaultElasticity(g, lam, MU, lf, device=local, precision="fp64", rtol=1e-12)
    K64 = eqd.stiffness_columns(fe64, cols[pick])[0]
    fe64.close()
    k_err = float(np.linalg.norm(Kmix[:, pick] - K64) / np.linalg.norm(K64))
    k_max = float(abs(Kmix[:, pick] - K64).max() / abs(K64).max())

    # Plain FP64 CG, one right-hand side at a time (the comparator).
    plain = eqd.FaultElasticity(g, lam, MU, lf, device=local, precision="fp64", chunk=1)
    nz = cols[np.abs(Kmix).sum(0) > 0]  # skip columns whose right-hand side is zero (ring nodes)
    sample = np.sort(rng.choice(nz, size=min(n_plain, len(nz)), replace=False)).astype(np.int32)
    eqd.stiffness_columns(plain, sample[:1])
    eqd.stiffness_columns(plain, sample[-1:])
    t0 = time.perf_counter()
    lat = []
    for c in sample:
        t1 = time.perf_counter()
        eqd.stiffness_columns(plain, [c])
        lat.append((time.perf_counter() - t1) * 1e3)
    plain_v = len(sample) / (time.perf_counter() - t0)
    plain.close()
    # Batched FP64 (same path) for context.
    b64 = eqd.FaultElasticity(g, lam, MU, lf, device=local, precision="fp64")
    bcols = cols if n_b64 is None or n_b64 >= len(cols) else cols[:n_b64]
    eqd.stiffness_columns(b64, bcols[:64])
    st64 = eqd._abi.Stats()
    eqd._abi.check(lib.eqd_stiffness_columns_device(
        b64.handle, eqd._abi.ptr(bcols), C.c_int32(len(bcols)), C.byref(b64.rs.opts()),
        C.c_void_p(kdev.data_ptr()), None, None, C.byref(st64)))
    batched64_v = len(bcols) / st64.device_seconds
    b64.close()

    # Sparse A of the workload's grid assembled on the GPU (the reference
    # assembles it with sparse Kronecker algebra before every solve).
    assembly = None
    if world == 1:
        fa = eqd.FaultElasticity(g, lam, MU, lf, device=local)
        t0 = time.perf_counter()
        Asp = eqd.assemble_operator(fa, "A")
        assembly = {"which": "A", "rows": int(Asp.shape[0]), "nnz": int(Asp.nnz),
                    "seconds": time.perf_counter() - t0, "what": "eqd_assemble to a host CSR (coloured probing)"}
        del Asp
        fa.close()

    serving = None
    if world == 1 and args.serve_requests > 0:
        serving = serving_leg(eqd, local, args.serve_requests, args.serve_rate)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        ofe, ref, ccols, nt = cpu_port_sample(args.config, n_cpu)
        ccols = np.intersect1d(ccols, cols) if args.config == "h25" else ccols
        Kc, itc, okc = ref.columns(ccols[:8], nthreads=nt, rtol=1e-13)
        pos = np.searchsorted(cols, ccols[:8])
        o_err = float(np.linalg.norm(Kmix[:, pos] - Kc) / np.linalg.norm(Kc)) if len(pos) and cols[pos[0]] == ccols[0] else None
        t0 = time.perf_counter()
        ref.columns(ccols, nthreads=nt)
        cdt = time.perf_counter() - t0
        cpu = {"value": len(ccols) / cdt, "unit": "columns/s", "cores": nt, "cpu_model": cpu_model(), "kind": "port",
               "sample": f"{len(ccols)} seeded columns of the workload, rtol 1e-10, OpenMP over columns "
                         "(C restatement of the reference column loop on the assembled CSR A)",
               "k_rel_err_vs_oracle_sample": o_err}

    line = {
        "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (unit slips; the workload is fully "
                                                          "determined by the grid)",
        "config": {"workload": wl, "columns": ncols, "precision": "mixed (FP32 CG, FP64 reliable updates)",
                   "rtol": opts.rtol, "parallelism": f"column shards x{world}",
                   "l2": "inputs larger than L2 (working set %.1f GB)" % (len(cols) * 6 * n1 * n23 * n23 * 24 / 1e9),
                   "mean_iterations": mean_it},
        "k_rel_err": {"frobenius_vs_fp64_rtol1e-12": k_err, "max_entry_vs_fp64_rtol1e-12": k_max,
                      "columns_checked": int(len(pick))},
        "step_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                    "what": "whole-K build time per step (all columns)"},
        "plain_fp64_single_rhs": {"value": plain_v, "unit": "columns/s",
                                  "latency_ms_p50": float(np.percentile(lat, 50)),
                                  "latency_ms_p99": float(np.percentile(lat, 99)),
                                  "sample": f"{len(sample)} columns solved one at a time"},
        "batched_fp64": {"value": batched64_v, "unit": "columns/s", "columns": int(len(bcols))},
        "speedup_vs_plain_fp64_single_rhs": value / plain_v,
        "speedup_vs_batched_fp64": value / batched64_v,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                     "peak_kind": peak_kind, "columns_per_launch": napply},
        "autotune": autotune,
        "chunk_tuning": chunk_tuning,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "wall_s_timed": wall,
    }
    if serving:
        line["serving"] = serving
    if assembly:
        line["assembly"] = assembly
    if gemv:
        line["gemv"] = gemv
    if gemm:
        line["batched_ks"] = gemm
    if toeplitz:
        line["toeplitz"] = toeplitz
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
