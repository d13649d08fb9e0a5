"""Served request stream: continuous batching of independent solves on one GPU.

The reference solves one model per process call (``StaticSolver.solve``,
gfem/solvers.py:481-605; ``_LinearSystem.solve``, gfem/solvers.py:396-474).  The
server keeps meshes resident and runs many requests at once:

* a *mesh entry* (:class:`MeshSpec` -> resident block, smoothed-aggregation
  hierarchy and mixed-precision solver, or a J2 model with its elastic
  hierarchy pinned) is set up once, by a set-up thread (host aggregation in a
  spawned process pool), and stays in HBM until it is evicted, least recently
  used first, to make room under the HBM budget;
* requests (:class:`SolveRequest`: a linear-elastic right-hand side, or a J2
  displacement-controlled step) queue in arrival order; ``slots`` worker threads,
  each with its own CUDA stream, take the oldest request whose entry is resident
  and idle, so requests that arrive while others are on the GPU start as soon as
  a slot and their mesh are free, and the kernels of different requests overlap
  on the device;
* a linear request is one FP32 matrix-free AMG-PCG inside FP64 iterative
  refinement (``NativeSolver.mixed``) to ``tol`` relative residual; a J2 request
  is a ``StaticSolver`` Newton solve with the mixed linear solver starting from
  the entry's pinned hierarchy.

Each result is the same alone and in the mix: every kernel and every reduction of
the path has a fixed summation order (fixed-point tile sums, fixed-order dot
products), so a request's arithmetic does not depend on what else runs.

An entry is used by one request at a time (its solver workspace and hierarchy
work vectors are per entry); requests for a busy entry wait while other entries'
requests proceed.
"""
import collections
import multiprocessing as mp
import threading
import time
from concurrent.futures import Future, ProcessPoolExecutor

import numpy as np
import torch

from . import linalg
from .materials import J2Plasticity, LinearElastic
from .model import Block, Model


class MeshSpec:
    """A mesh with its material and prescribed-DOF mask; ``key`` names the entry.

    X (nn, 3), conn (ne, nnode), etype HEX8 / TET10, material LinearElastic or
    J2Plasticity, fixed (3 nn,) bool (prescribed value zero for linear requests)."""

    def __init__(self, key, X, conn, etype, material, fixed):
        self.key = key
        self.X = np.ascontiguousarray(np.asarray(X, dtype=np.float64))
        self.conn = np.ascontiguousarray(np.asarray(conn, dtype=np.int32))
        self.etype, self.material = etype, material
        self.fixed = np.asarray(fixed, dtype=bool).reshape(-1)
        self.ndof = 3 * len(self.X)
        if self.fixed.size != self.ndof:
            raise ValueError("fixed mask must hold 3 entries per node")

    @property
    def j2(self):
        return isinstance(self.material, J2Plasticity)

    def device_bytes_estimate(self):
        """Upper estimate of the HBM an entry holds: element streams, index maps,
        hierarchy (operator complexity below 1.6 of a 3x3-block fine matrix that is
        not stored) and solver vectors."""
        ne, nd = len(self.conn), self.ndof
        per_el = 420 if self.etype.name == "C3D10" else 360
        return int(ne * per_el + nd * 81 * 12 * 0.6 + nd * 8 * 24 + (ne * self.etype.ngp * 19 * 16 if self.j2 else 0))


class SolveRequest:
    """One solve.  Linear: ``rhs`` (3 nn,) nodal forces.  J2: ``step`` (a
    :class:`solvers.Step`).  Timing fields are filled in by the server."""

    _ids = iter(range(1 << 62))

    def __init__(self, spec, rhs=None, step=None):
        if (rhs is None) == (step is None):
            raise ValueError("give a right-hand side (linear) or a step (J2)")
        if step is not None and not spec.j2:
            raise ValueError("a step request needs a J2 mesh entry")
        if rhs is not None and spec.j2:
            raise ValueError("a right-hand-side request needs a linear-elastic mesh entry")
        self.id = next(self._ids)
        self.spec, self.rhs, self.step = spec, rhs, step
        self.t_arrival = self.t_start = self.t_done = None
        self.info = {}

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrival


def _host_setup(args):
    """Aggregation set-up of one entry from its element stiffness (worker process)."""
    dofs, Ke, ndof, free, X = args
    A = linalg.bc_matrix(linalg.ops_assemble([(dofs, Ke)], ndof), free)
    h = linalg.amg_setup(A, X)
    if h["levels"]:
        h["levels"][0]["A"] = None          # level 0 is smoothed with the matrix-free product
    return h


class _Entry:
    def __init__(self, spec, setup, graph=True, amg=None):
        self.spec = spec
        self.amg = amg if amg is not None else linalg.AMG.from_setup(setup)
        if spec.j2:
            self.model = Model(spec.X)
            self.model.add_block(spec.conn, spec.etype, spec.material)
            self.block, self.solver = self.model.blocks[0], None
        else:
            self.model = None
            self.block = Block(spec.conn, spec.etype, spec.material, X=spec.X)
            self.block.set_fixed(spec.fixed)
            self.solver = linalg.NativeSolver(self.block, "mf32", "amg", self.amg, graph=graph)
        self.static = None              # the J2 entry's StaticSolver, made by its first request
        self.bytes = spec.device_bytes_estimate()
        self.busy = False
        self.last_used = time.time()


class SolveServer:
    """Continuous-batching solve server (see the module docstring).

    slots: requests in flight at once; hbm_budget: bytes of resident entries;
    tol: relative residual of linear requests (FP64 refinement); amg_setup:
    "device" (the hierarchy is set up on the GPU by the set-up thread,
    linalg.DeviceAMG) or "host" (host aggregation set-up in ``setup_workers``
    spawned processes, 0: in the set-up thread).
    ``solve_fn(entry, request)`` replaces the device solve (host-side tests)."""

    def __init__(self, slots=8, hbm_budget=150e9, tol=1e-8, inner_tol=2e-5, setup_workers=4, graph=True,
                 solve_fn=None, setup_fn=None, amg_setup="device"):
        if amg_setup not in ("device", "host"):
            raise ValueError(f"unknown AMG set-up {amg_setup!r}")
        self.slots, self.budget, self.tol, self.inner_tol = slots, float(hbm_budget), tol, inner_tol
        self.graph = graph
        self.amg_setup = amg_setup
        self._solve_fn = solve_fn or self._device_solve
        self._setup_fn = setup_fn or self._device_setup
        self._cv = threading.Condition()
        self._pending = collections.deque()
        self._waiting = collections.Counter()           # mesh key -> pending requests (no scans of a long backlog)
        self._waiting_spec = {}                          # mesh key -> its spec, while it has pending requests
        self._entries = collections.OrderedDict()       # key -> _Entry (LRU order)
        self._setting_up = set()
        self._futures = {}
        self._stop = False
        self.resident_bytes = 0
        self.completed = []
        self.evictions = 0
        self._pool = (ProcessPoolExecutor(max_workers=setup_workers, mp_context=mp.get_context("spawn"))
                      if setup_workers and setup_fn is None and amg_setup == "host" else None)
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(slots)]
        self._threads.append(threading.Thread(target=self._setup_loop, daemon=True))
        for t in self._threads:
            t.start()

    # ------------------------------------------------------------------ API
    def submit(self, req):
        """Queue a request; returns a Future resolving to (x on the host, info)."""
        fut = Future()
        with self._cv:
            if self._stop:
                raise RuntimeError("server is closed")
            req.t_arrival = time.perf_counter()
            self._futures[req.id] = fut
            self._pending.append(req)
            self._hold(req)
            self._cv.notify_all()
        return fut

    def cancel(self, req):
        """Withdraw a request that has not started; its future raises
        CancelledError.  Returns False when it already runs or has finished."""
        with self._cv:
            if req not in self._pending:
                return False
            self._pending.remove(req)
            self._release(req)
            fut = self._futures.pop(req.id)
        fut.cancel()
        return True

    def cancel_pending(self):
        """Withdraw every request that has not started (e.g. the backlog at the end
        of a measurement window); returns how many were withdrawn."""
        with self._cv:
            reqs = list(self._pending)
            self._pending.clear()
            self._waiting.clear()
            self._waiting_spec.clear()
            futs = [self._futures.pop(r.id) for r in reqs]
        for f in futs:
            f.cancel()
        return len(reqs)

    def warm(self, specs):
        """Set up entries ahead of the stream (blocks until they are resident)."""
        for sp in specs:
            with self._cv:
                if sp.key in self._entries or sp.key in self._setting_up:
                    continue
            self._make_entry(sp)

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join(timeout=60)
        if self._pool is not None:
            self._pool.shutdown()
        with self._cv:
            self._entries.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def entry(self, key):
        with self._cv:
            return self._entries.get(key)

    def _hold(self, req):
        k = req.spec.key
        self._waiting[k] += 1
        self._waiting_spec[k] = req.spec

    def _release(self, req):
        k = req.spec.key
        self._waiting[k] -= 1
        if self._waiting[k] <= 0:
            del self._waiting[k]
            self._waiting_spec.pop(k, None)

    # ------------------------------------------------------------------ set-up
    def _device_setup(self, spec):
        blk = Block(spec.conn, spec.etype, LinearElastic(spec.material.E, spec.material.nu), X=spec.X)
        Ke = blk.stiffness(torch.zeros(spec.ndof, dtype=torch.float64, device="cuda"), blk.init_state())
        if self.amg_setup == "device":
            blk.set_fixed(spec.fixed)
            amg = linalg.DeviceAMG(blk, Ke)
            del blk, Ke
            return _Entry(spec, None, self.graph, amg=amg)
        dofs = (spec.conn.astype(np.int64)[:, :, None] * 3 + np.arange(3)).reshape(len(spec.conn), -1)
        job = (dofs, Ke.cpu().numpy(), spec.ndof, (~spec.fixed).astype(np.float64), spec.X)
        del blk, Ke
        setup = self._pool.submit(_host_setup, job).result() if self._pool is not None else _host_setup(job)
        return _Entry(spec, setup, self.graph)

    def _make_entry(self, spec):
        """Set up spec's entry under the HBM budget (evicting idle entries, least
        recently used first); returns the entry."""
        need = spec.device_bytes_estimate()
        with self._cv:
            while self.resident_bytes + need > self.budget:
                victim = next((k for k, e in self._entries.items()
                               if not e.busy and not self._waiting[k]), None)
                if victim is None:
                    if not self._entries:
                        break                                 # an entry larger than the budget runs alone
                    self._cv.wait(0.05)
                    continue
                self.resident_bytes -= self._entries.pop(victim).bytes
                self.evictions += 1
            self._setting_up.add(spec.key)
        try:
            e = self._setup_fn(spec)
        finally:
            with self._cv:
                self._setting_up.discard(spec.key)
        with self._cv:
            self._entries[spec.key] = e
            self.resident_bytes += e.bytes
            self._cv.notify_all()
        return e

    def _setup_loop(self):
        if torch.cuda.is_available() and self._setup_fn == self._device_setup:
            torch.cuda.set_stream(torch.cuda.Stream())       # keep set-up work off the default stream
        while True:
            with self._cv:
                spec = None
                while spec is None:
                    if self._stop:
                        return
                    spec = next((sp for k, sp in self._waiting_spec.items()
                                 if k not in self._entries and k not in self._setting_up), None)
                    if spec is None:
                        self._cv.wait(0.05)
            try:
                self._make_entry(spec)
            except Exception as exc:                                  # fail the requests of this mesh
                with self._cv:
                    for r in [r for r in self._pending if r.spec.key == spec.key]:
                        self._pending.remove(r)
                        self._release(r)
                        self._futures.pop(r.id).set_exception(exc)

    # ------------------------------------------------------------------ solving
    def _device_solve(self, entry, req):
        spec = req.spec
        if not spec.j2:
            b = torch.as_tensor(np.asarray(req.rhs, dtype=np.float64), device="cuda")
            x, k, p, rel = entry.solver.mixed(b, tol=self.tol, inner_tol=self.inner_tol)
            if not np.isfinite(rel) or rel > 10 * self.tol:
                raise RuntimeError(f"request {req.id}: refinement did not converge (rel. residual {rel:.2e})")
            return x.cpu().numpy(), dict(iters=k, passes=p, relres=rel)
        from .solvers import StaticSolver
        if entry.static is None:        # kept with the entry: its solver handle and captured graphs are reused
            entry.static = StaticSolver(entry.model, rtol=1e-6, linear_solver="mixed", tangent="mf", cg_tol=1e-6,
                                        verbose=False, graph=self.graph, amg=entry.amg)
        u, states, info = entry.static.solve(req.step)
        return u.cpu().numpy(), dict(newton=info["iterations"], increments=info["increments"])

    def _worker(self, slot):
        stream = torch.cuda.Stream() if torch.cuda.is_available() and self._solve_fn == self._device_solve else None
        while True:
            with self._cv:
                req = None
                while req is None:
                    if self._stop:
                        return
                    for r in self._pending:
                        e = self._entries.get(r.spec.key)
                        if e is not None and not e.busy:
                            req, entry = r, e
                            break
                    if req is None:
                        self._cv.wait(0.05)
                self._pending.remove(req)
                self._release(req)
                entry.busy = True
                entry.last_used = time.time()
                self._entries.move_to_end(req.spec.key)
                fut = self._futures.pop(req.id)
            req.t_start = time.perf_counter()
            try:
                if stream is not None:
                    with torch.cuda.stream(stream):
                        x, info = self._solve_fn(entry, req)
                        stream.synchronize()
                else:
                    x, info = self._solve_fn(entry, req)
                req.t_done = time.perf_counter()
                req.info = dict(info, slot=slot)
                ok, result = True, (x, req.info)
            except Exception as exc:
                req.t_done = time.perf_counter()
                ok, result = False, exc
            with self._cv:
                entry.busy = False
                self.completed.append(req)
                self._cv.notify_all()
            if ok:
                fut.set_result(result)
            else:
                fut.set_exception(result)


def request_records(reqs):
    """One JSON-ready record per finished request: id, mesh key, kind, DOF, arrival
    to start (queue) and start to done (service) times, latency, and the solver's info
    (iterations, passes, relative residual, slot) — the raw data behind p50 / p99."""
    out = []
    for r in reqs:
        if r.t_done is None:
            continue
        info = {k: (v.item() if hasattr(v, "item") else v) for k, v in r.info.items()
                if isinstance(v, (int, float, str, bool, np.integer, np.floating))}
        out.append(dict(id=int(r.id), mesh=r.spec.key, kind="j2" if r.spec.j2 else "linear", ndof=int(r.spec.ndof),
                        queue_s=float(r.t_start - r.t_arrival) if r.t_start is not None else None,
                        service_s=float(r.t_done - r.t_start) if r.t_start is not None else None,
                        latency_s=float(r.latency), **info))
    return out


def latency_stats(reqs):
    """p50 / p99 latency (s), throughput (completed / makespan) of finished requests."""
    lat = np.array([r.latency for r in reqs if r.latency is not None])
    if not len(lat):
        return dict(n=0)
    t0 = min(r.t_arrival for r in reqs)
    t1 = max(r.t_done for r in reqs)
    return dict(n=len(lat), p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)),
                mean_s=float(lat.mean()), solves_per_s=float(len(lat) / max(t1 - t0, 1e-9)))
