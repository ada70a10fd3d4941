"""Serving stiffness-column requests with continuous batching.

The reference builds all of K in one blocking call (`fault_stiffness`,
src/FaultResponse.jl:229-287). `Server` answers requests for any subset of
K's columns (the work of `run_columns!`, :244-263), on several grids, as they
arrive:

    srv = Server(hbm_budget_bytes=150e9)
    srv.add(fe, slots=256)             # fe: FaultElasticity (owned by srv now)
    req = srv.submit(fe, [0, 17, 300]) # returns at once
    K_cols = req.result(timeout=60)    # 2nf x 3, FP64

Each attached grid keeps a pool of CG slots resident in HBM (operator tables,
Krylov vectors, per-column state). Columns of queued requests enter free
slots as earlier columns finish, beside columns of other requests on the
same grid; different grids run at the same time on their own CUDA streams.
The server's worker is a native thread inside libeqd (include/eqd.h,
`eqd_server_*`); this module only wraps it.
"""
import ctypes as C
import time

import numpy as np

from . import _abi
from ._abi import EqdArgumentError, check, lib, ptr

STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


class Request:
    """A submitted request; `result()` waits for and returns its K columns."""

    def __init__(self, server, rid, fe, cols, out):
        self._srv, self.id, self.fe, self.cols, self._out = server, rid, fe, cols, out

    def done(self):
        d = C.c_int32()
        check(lib().eqd_server_poll(self._srv.handle, C.c_int64(self.id), C.byref(d)))
        return bool(d.value)

    def wait(self, timeout=None):
        t = -1.0 if timeout is None else float(timeout)
        check(lib().eqd_server_wait(self._srv.handle, C.c_int64(self.id), C.c_double(t)))

    def result(self, timeout=None):
        self.wait(timeout)
        return self._out

    def info(self):
        i = _abi.RequestInfo()
        check(lib().eqd_server_request_info(self._srv.handle, C.c_int64(self.id), C.byref(i)))
        return dict(state=STATES.get(i.state, i.state), ncols=i.ncols, unconverged=i.unconverged,
                    iterations=i.iterations, max_iterations=i.max_iterations, t_submit=i.t_submit,
                    t_start=i.t_start, t_done=i.t_done,
                    latency=(i.t_done - i.t_submit) if i.t_done >= 0 else None)

    def release(self):
        check(lib().eqd_server_release(self._srv.handle, C.c_int64(self.id)))


class Server:
    """`eqd_server`: solver options shared by every grid (`precision`,
    `rtol`, ...; the same keywords as `CGSolver`), slot pools within
    `hbm_budget_bytes` (0: free device memory minus 2 GiB)."""

    def __init__(self, hbm_budget_bytes=0, rtol=1e-10, atol=0.0, itmax=0, precision="mixed", reliable_delta=0.01,
                 split=True, precond="none"):
        o = _abi.default_opts()
        o.rtol, o.atol, o.itmax = float(rtol), float(atol), int(itmax)
        if precond not in ("none", "jacobi"):
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"precond must be :none or :jacobi, got {precond}")
        o.precond = _abi.EQD_PRECOND_JACOBI if precond == "jacobi" else _abi.EQD_PRECOND_NONE
        if precision not in ("mixed", "fp64"):
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"precision must be 'mixed' or 'fp64', got {precision}")
        o.precision = _abi.EQD_PREC_MIXED if precision == "mixed" else _abi.EQD_PREC_FP64
        o.reliable_delta = float(reliable_delta)
        if not split:
            o.flags |= _abi.EQD_FLAG_NO_SPLIT
        h = C.c_void_p()
        check(lib().eqd_server_create(C.byref(o), C.c_uint64(int(hbm_budget_bytes)), C.byref(h)))
        self._h = h
        self._grids = []

    @property
    def handle(self):
        if self._h is None:
            raise _abi.EqdError(_abi.EQD_ERR_ARG, "server was closed")
        return self._h

    def add(self, fe, slots=0):
        """Attach a grid with `slots` CG slots (0: as many as the budget
        allows, at most 512). The grid belongs to the server until close()."""
        check(lib().eqd_server_add_grid(self.handle, fe.handle, C.c_int32(slots)))
        self._grids.append(fe)

    def submit(self, fe, cols):
        """Queue K columns `cols` of an attached grid; returns a Request."""
        cc = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.empty((2 * fe.nf, len(cc)), order="F")
        rid = C.c_int64()
        check(lib().eqd_server_submit(self.handle, fe.handle, ptr(cc), C.c_int32(len(cc)),
                                      out.ctypes.data_as(C.c_void_p), C.byref(rid)))
        return Request(self, rid.value, fe, cc, out)

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().eqd_server_destroy(self._h)
            self._h = None
            self._grids = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_arrivals(rate, duration, rng):
    """Arrival times of a Poisson process of `rate` per second over `duration` s."""
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.array(out)
        out.append(t)


def run_mix(server, grids, weights, rate, nreq, rng, max_rhs=512, timeout=600.0):
    """Open-loop load: `nreq` requests at Poisson `rate` req/s; each picks a
    grid by `weights` and ⌊exp(U(0, ln max_rhs))⌋ + 1 (≤ max_rhs) seeded
    unit-slip columns. Returns (requests, wall seconds)."""
    w = np.asarray(weights, dtype=float) / np.sum(weights)
    gaps = rng.exponential(1.0 / rate, size=nreq)
    reqs = []
    t0 = time.perf_counter()
    due = t0
    for k in range(nreq):
        due += gaps[k]
        g = grids[rng.choice(len(grids), p=w)]
        n = min(int(np.floor(np.exp(rng.uniform(0.0, np.log(max_rhs))))) + 1, max_rhs, 2 * g.nf)
        cols = rng.choice(2 * g.nf, size=n, replace=False)
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        reqs.append(server.submit(g, cols))
    for r in reqs:
        r.wait(timeout)
    return reqs, time.perf_counter() - t0
