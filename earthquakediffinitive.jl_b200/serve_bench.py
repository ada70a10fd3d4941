"""Serving benchmark: Poisson arrivals of stiffness-column requests over the
BP8 grids, answered by the continuous-batching server.

    python earthquakediffinitive.jl_b200/serve_bench.py [--rates 10,100,1000] [--requests 200]

Mix: each request names a grid h in {100, 50, 25, 20} m with weights
0.4/0.3/0.2/0.1 and carries floor(exp(U(0, ln 512))) + 1 unit-slip columns
(at most 512) at uniformly drawn fault nodes (seed 5); K columns come back in
FP64. Slot pools are sized within a 150 GB HBM budget. Prints one JSON line
per arrival rate: p50/p99 request latency (submit -> last column delivered),
columns/s over the run, and the K error of a sample of requests against a
tight FP64 build of the same columns (checked after the timed run).

Grids (`build_model`, src/BP8.jl:196-206, Omega_f = the whole fault plane):
  h = 100 m: L_fault 800, L_normal 800  ->  9 x 17 x 17 per side
  h =  50 m: L_fault 800, L_normal 400  ->  9 x 33 x 33
  h =  25 m: L_fault 1600, L_normal 800 -> 33 x 129 x 129
  h =  20 m: L_fault 800, L_normal 400  -> 21 x 81 x 81
"""
import argparse
import importlib.util
import json
import os
import sys
import time

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
GRIDS = {  # h: (dz, L_fault, L_normal, weight, slots)
    100: (100.0, 800.0, 800.0, 0.4, 512),
    50: (50.0, 800.0, 400.0, 0.3, 512),
    25: (25.0, 1600.0, 800.0, 0.2, 512),
    20: (20.0, 800.0, 400.0, 0.1, 512),
}
MU = 32.04e9


def _package():
    if "eqd_b200" in sys.modules:
        return sys.modules["eqd_b200"]
    spec = importlib.util.spec_from_file_location(
        "eqd_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["eqd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="10,30,100,300,1000")
    ap.add_argument("--requests", type=int, default=200, help="requests per rate")
    ap.add_argument("--grids", default="100,50,25,20")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--check", type=int, default=6, help="requests per rate checked against FP64")
    ap.add_argument("--seed", type=int, default=5)
    a = ap.parse_args(argv)
    eqd = _package()
    from eqd_b200.serving import run_mix

    hs = [int(h) for h in a.grids.split(",")]
    lam = eqd.lame_lambda(MU, 0.25)
    srv = eqd.Server(hbm_budget_bytes=int(a.budget_gb * 1e9))
    fes, weights = [], []
    t0 = time.perf_counter()
    for h in hs:
        dz, Lf, Ln, w, slots = GRIDS[h]
        fe = eqd.FaultElasticity(eqd.bp8_grids(dz, Lf, Ln), lam, MU, Lf)
        srv.add(fe, slots=slots)
        fe.h = h
        fes.append(fe)
        weights.append(w)
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(a.seed)
    # Warm-up: one small request per grid (first graph launches, page-in).
    for fe in fes:
        srv.submit(fe, [0]).wait(600)
    results = []
    for rate in [float(r) for r in a.rates.split(",")]:
        reqs, wall = run_mix(srv, fes, weights, rate, a.requests, rng)
        infos = [r.info() for r in reqs]
        lat = np.array([i["latency"] for i in infos]) * 1e3
        ncols = int(sum(i["ncols"] for i in infos))
        span = max(i["t_done"] for i in infos) - min(i["t_submit"] for i in infos)
        by_grid = {}
        for r, i in zip(reqs, infos):
            by_grid.setdefault(r.fe.h, []).append(i["latency"] * 1e3)
        line = {
            "metric": "serving: request latency and K columns/s (continuous batching, Poisson arrivals)",
            "rate_req_s": rate, "requests": len(reqs), "columns": ncols,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "latency_ms_p50_by_grid_h": {str(h): float(np.percentile(v, 50)) for h, v in sorted(by_grid.items())},
            "columns_per_s": ncols / span, "offered_s": wall, "unconverged": int(sum(i["unconverged"] for i in infos)),
            "grids_h_m": hs, "weights": weights, "hbm_budget_gb": a.budget_gb,
        }
        results.append((line, reqs))
    setup = {"setup_s": setup_s}
    srv.close()
    # Accuracy: sampled requests against a tight FP64 build of the same columns.
    chk_fe = {}
    for line, reqs in results:
        errs = []
        for r in reqs[: a.check]:
            h = r.fe.h
            if h not in chk_fe:
                dz, Lf, Ln, _, _ = GRIDS[h]
                chk_fe[h] = eqd.FaultElasticity(eqd.bp8_grids(dz, Lf, Ln), lam, MU, Lf, precision="fp64", rtol=1e-12)
            K64 = eqd.stiffness_columns(chk_fe[h], r.cols)[0]
            K = r._out  # filled before the request completed (the server is closed now)
            errs.append(float(np.linalg.norm(K - K64) / np.linalg.norm(K64)))
        line["k_rel_err_vs_fp64_max"] = max(errs) if errs else None
        line["k_rel_err_sample_requests"] = len(errs)
        line.update(setup)
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
