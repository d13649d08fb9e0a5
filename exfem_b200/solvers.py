"""Quasi-static Newton procedure over the device hot path (drop-in for the
``StaticSolver`` part of ``gfem.solvers``).

* ``Monitor``, ``Step``, ``State`` — gfem/solvers.py:24-95 (the fields the
  static procedure uses).
* ``_Setup`` — gfem/solvers.py:104-217 for MPC-free, amplitude-free steps:
  fixed mask, prescribed values ramped from the step's start state, load groups
  summed with ``np.add.at``, precomputed load vectors (``dloads``).
* ``_LinearSystem`` — gfem/solvers.py:235-477.  Methods:
    "direct"  host sparse LU of the assembled tangent (a reference solver);
    "amg"     plain FP64 path: FP64 operator (stored Ke, or matrix-free with
              ``tangent="mf"``) + FP64 AMG V-cycle, PCG in the library;
    "jacobi"  FP64 operator + Jacobi PCG;
    "cheby"   FP64 operator + the set-up-free Chebyshev-Jacobi polynomial
              preconditioner (degree 6, bound by device power iteration,
              gfem/solvers.py:289-306, 328-342);
    "mixed"   FP32 matrix-free operator + FP32 V-cycle (FP64 coarse solve)
              inside FP64 iterative refinement with an FP64 matrix-free residual
              (solvers.py:344-384);
    "auto"    direct up to 20000 DOFs, else amg (the reference's GPU rule).
  The hierarchy is built on the first solve of a step from the assembled FP64
  tangent, frozen across Newton iterations and increments, and rebuilt when the
  PCG iteration count exceeds 4x the first one (solvers.py:442-470); level 0 is
  always smoothed with the current operator (solvers.py:311-314).  For "amg" on
  models of at least ``async_amg`` DOFs (150000, the reference's threshold) the
  hierarchy is set up in a background thread on its own CUDA stream while the
  solves run Chebyshev-Jacobi PCG (solvers.py:445-464).
* ``StaticSolver`` — gfem/solvers.py:481-683: automatic incrementation (x1.5
  growth after <= 5 iterations, x0.25 cutback), tangent predictor, Newton with
  the reference convergence test and a 4-step backtracking line search.

``tangent="ebe"`` stores element tangents Ke (the reference default);
``tangent="mf"`` (alias "jvp") keeps the tangent matrix-free: the force kernel
leaves per-Gauss-point consistent-tangent data in HBM and every product is
evaluated element by element (the B200 replacement of ``Model.tangent_jvp``).
"""
import time

import numpy as np
import torch

from . import linalg
from .linalg import NativeSolver


class Monitor:                                                          # solvers.py:24-45
    def __init__(self, verbose=True):
        self.verbose = verbose
        self.stop = False

    def log(self, msg):
        if self.verbose:
            print(msg, flush=True)

    def iteration(self, **kw):
        pass

    def increment(self, **kw):
        pass

    def frame(self, t, u, states, **kw):
        pass

    def should_stop(self):
        return self.stop


class Step:                                                             # solvers.py:48-80
    def __init__(self, name="Step-1", kind="static", time_period=1.0, dt_init=None, dt_min=None, dt_max=None,
                 max_inc=1000, bcs=(), loads=(), dloads=(), **kw):
        self.name, self.kind, self.T = name, kind, float(time_period)
        self.dt_init = dt_init or self.T
        self.dt_min = dt_min if dt_min is not None else 1e-5 * self.T
        self.dt_max = dt_max or self.T
        self.max_inc = max_inc
        self.bcs, self.loads, self.dloads = list(bcs), list(loads), list(dloads)
        self.output_every = kw.get("output_every", 1)


class State:                                                            # solvers.py:83-95
    def __init__(self, model):
        self.u = torch.zeros(model.ndof, dtype=torch.float64, device="cuda")
        self.states = model.init_state()
        self.fext = torch.zeros(model.ndof, dtype=torch.float64, device="cuda")
        self.time = 0.0
        self.reactions = torch.zeros(model.ndof, dtype=torch.float64, device="cuda")


def _ramp(t, T):                                                        # solvers.py:220-221
    return min(max(t / T, 0.0), 1.0) if T > 0 else 1.0


class _Setup:                                                           # solvers.py:104-217
    def __init__(self, model, step, state):
        nd = model.ndof
        self.step = step
        self.fixed = np.zeros(nd, bool)
        self.target = np.zeros(nd)
        for bc in step.bcs:
            nodes, dof, val = bc[:3]
            d = model.dof(nodes, dof)
            self.fixed[d] = True
            self.target[d] = val
        # point loads summed on the host (few entries), distributed load vectors
        # summed on the device; masks and targets scattered on the device from the
        # prescribed DOFs, so only index-sized arrays and the load vectors cross PCIe
        g = torch.zeros(nd, dtype=torch.float64, device="cuda")
        if step.loads:
            gp = np.zeros(nd)
            for ld in step.loads:
                nodes, dof, val = ld[:3]
                np.add.at(gp, model.dof(nodes, dof), val)
            nz = np.nonzero(gp)[0]
            g[torch.as_tensor(nz, device="cuda")] = torch.as_tensor(gp[nz], device="cuda")
        for dl in step.dloads:
            vec = dl[0] if isinstance(dl, (tuple, list)) else dl
            g += torch.as_tensor(np.asarray(vec, float) if not isinstance(vec, torch.Tensor) else vec,
                                 dtype=torch.float64, device="cuda").reshape(-1)
        self.group = g
        self.fprev = state.fext
        self.ustart = state.u.clone()
        idx = np.nonzero(self.fixed)[0]
        idx_j = torch.as_tensor(idx, device="cuda")
        self.fixed_j = torch.zeros(nd, dtype=torch.bool, device="cuda")
        self.fixed_j[idx_j] = True
        self.target_j = torch.zeros(nd, dtype=torch.float64, device="cuda")
        self.target_j[idx_j] = torch.as_tensor(self.target[idx], device="cuda")
        self.free = (~self.fixed_j).to(torch.float64)
        self._free_np = None

    @property
    def free_np(self):
        if self._free_np is None:
            self._free_np = (~self.fixed).astype(float)
        return self._free_np

    def fext(self, t):
        r = _ramp(t, self.step.T)
        return self.fprev * (1 - r) + self.group * r

    def fext_final(self):
        return self.fext(self.step.T)

    def prescribed(self, t):
        r = _ramp(t, self.step.T)
        tgt = self.ustart + (self.target_j - self.ustart) * r
        return torch.where(self.fixed_j, tgt, torch.zeros_like(tgt))


class _LinearSystem:                                                    # solvers.py:235-477
    """Solves (free K free + fixed I) x = b with the chosen back-end."""

    def __init__(self, model, method="auto", tangent="ebe", cg_tol=1e-9, cg_maxiter=20000, monitor=None,
                 graph=True, amg_setup="auto", mixed_mode="reliable", operator="gather", async_amg=150000):
        self.m = model
        self.async_amg = async_amg              # DOFs from which "amg" sets up in the background (None: never)
        self._amg_future = None
        self._pool = None
        if operator not in ("gather", "csr"):
            raise ValueError(f"unknown operator {operator!r}")
        # stored-Ke operator of the "amg" / "jacobi" methods with tangent="ebe":
        # "gather" = element-by-element products, "csr" = the element matrices
        # assembled on the device into one CSR matrix (gfem/solvers.py:239-247, 406-412)
        self.operator = operator
        self.mixed_mode = mixed_mode            # linalg.NativeSolver: "reliable" or "restart"
        if amg_setup not in ("auto", "host", "device"):
            raise ValueError(f"unknown AMG set-up {amg_setup!r}")
        # where the hierarchy is set up: "host" (assembled CSR, host set-up),
        # "device" (linalg.DeviceAMG: the same hierarchy, assembled and multiplied
        # on the GPU); "auto" = device
        self.amg_setup = amg_setup
        if method == "auto":
            method = "direct" if model.ndof <= 20000 else "amg"
        if method not in ("direct", "amg", "jacobi", "mixed", "cheby"):
            raise ValueError(f"unknown linear solver {method!r}")
        self.method = method
        self.tangent = "mf" if tangent in ("mf", "jvp") or method == "mixed" else "ebe"
        self.cg_tol, self.cg_maxiter = cg_tol, cg_maxiter
        self.mon = monitor or Monitor(False)
        self.graph = graph
        self.pinned_amg = None                # a hierarchy every step starts from (served solves)
        self.amg = None
        self.amg_iters0 = None
        self.last_iters = 0
        self.last_passes = 0
        self.last_setup_time = 0.0
        self._solvers = {}

    def reset(self):
        if self._amg_future is not None:                 # a background set-up of the previous step
            self._amg_future.result()
            self._amg_future = None
        self.amg = self.pinned_amg
        self.amg_iters0 = None
        # solvers over a pinned hierarchy stay (with their captured graphs and the FP32
        # pass tolerance their first mixed solve measured)
        self._solvers = {k: v for k, v in self._solvers.items() if self.amg is not None and k[2] == id(self.amg)}

    def _solver(self, op, pc):
        key = (op, pc, id(self.amg))
        s = self._solvers.get(key)
        if s is None:
            s = NativeSolver(self.m.blocks, op, pc, self.amg if pc == "amg" else None, graph=self.graph,
                             mixed_mode=self.mixed_mode)
            self._solvers = {k: v for k, v in self._solvers.items() if k[2] == id(self.amg)}
            self._solvers[key] = s
        return s

    def assemble(self, ops, setup):
        A = linalg.ops_assemble(ops, self.m.ndof)
        return linalg.bc_matrix(A, setup.free_np)

    def _setup_ops(self, ops, ctx):
        """Element tangents for assembly: the stored ops, or a stiffness evaluation at
        the matrix-free operator's state."""
        if isinstance(ops, list):
            return ops
        u, s, fields = ctx
        return self.m.stiffness_ops(u, s, fields)

    def _build_amg(self, ops, setup, ctx):
        t0 = time.time()
        where = self.amg_setup
        if where == "auto":
            where = "device"
        if where == "device":
            Kes = [K for _, K in self._setup_ops(ops, ctx)]
            self.amg = linalg.DeviceAMG(self.m.blocks, Kes)
        else:
            A = self.assemble(self._setup_ops(ops, ctx), setup)
            self.amg = linalg.AMG(A, self.m.X)
        self.amg_iters0 = None
        self._solvers = {}
        self.last_setup_time = time.time() - t0
        self.mon.log(f"    {self.amg.info()}  setup {self.last_setup_time:.2f}s")

    def _start_background_build(self, ops, setup, ctx):
        """Set the hierarchy up in a worker thread on its own stream, from element
        matrices evaluated now on the calling stream."""
        import concurrent.futures as cf
        Kes = [K for _, K in self._setup_ops(ops, ctx)]
        ready = torch.cuda.Event()
        ready.record()
        device = torch.cuda.current_device()
        where = "device" if self.amg_setup == "auto" else self.amg_setup
        host_A = self.assemble(list(zip([b.dofs() for b in self.m.blocks], Kes)), setup) if where == "host" else None

        def build():
            t0 = time.time()
            torch.cuda.set_device(device)
            side = torch.cuda.Stream()
            with torch.cuda.stream(side):
                side.wait_event(ready)
                amg = linalg.DeviceAMG(self.m.blocks, Kes) if host_A is None else linalg.AMG(host_A, self.m.X)
            side.synchronize()
            return amg, time.time() - t0

        self._pool = self._pool or cf.ThreadPoolExecutor(1)
        self._amg_future = self._pool.submit(build)
        self.mon.log("    AMG set-up started in the background; Chebyshev-Jacobi PCG meanwhile")

    def _collect_background_build(self):
        fut = self._amg_future
        if fut is not None and fut.done():
            self._amg_future = None
            self.amg, self.last_setup_time = fut.result()
            self.amg_iters0 = None
            self._solvers = {}
            self.mon.log(f"    {self.amg.info()}  (set up in the background, {self.last_setup_time:.2f}s)")

    def _pcg(self, ops, b, op, pc):
        S = self._solver(op, pc)
        if op in ("ebe64", "csr64"):
            S.set_ke([K for _, K in ops])
        return S.pcg(b, tol=self.cg_tol, maxiter=self.cg_maxiter)

    def solve(self, ops, b, setup, jvp_args=None, rebuild=False):
        """ops: [(dofs, Ke)] (tangent="ebe") or None with jvp_args = (u, states, fields)
        (tangent="mf"; the block's tangent data must be current)."""
        for blk in self.m.blocks:
            blk.set_fixed(setup.fixed)
        b = b.to(torch.float64)
        if self.method == "direct":
            A = self.assemble(self._setup_ops(ops, jvp_args), setup)
            x = linalg.Direct(A).solve(b.cpu().numpy())
            self.last_iters = 1
            return torch.as_tensor(x, device="cuda")
        op = ("csr64" if self.operator == "csr" else "ebe64") if self.tangent == "ebe" else "mf64"
        if self.method == "amg":
            self._collect_background_build()
            if (self.amg is None or rebuild) and self._amg_future is None:
                if self.async_amg is not None and self.m.ndof >= self.async_amg:
                    self._start_background_build(ops, setup, jvp_args)
                else:
                    self._build_amg(ops, setup, jvp_args)
            if self.amg is None or (rebuild and self._amg_future is not None):
                x, k, rr = self._pcg(ops, b, op, "cheby")
                self.last_iters = k
                return x
        if self.method == "mixed" and (self.amg is None or rebuild):
            self._build_amg(ops, setup, jvp_args)
        if self.method == "mixed":
            S = self._solver("mf32", "amg")
            x, k, p, rel = S.mixed(b, tol=self.cg_tol, maxiter=self.cg_maxiter)
            self.last_iters, self.last_passes = k, p
            if not np.isfinite(rel) or rel > max(self.cg_tol * 10, 1e-3):
                self.mon.log(f"    warning: mixed refinement not converged ({k} it, {p} passes, rel.res {rel:.2e})")
            return x
        pc = self.method if self.method in ("jacobi", "cheby") else "amg"
        x, k, rr = self._pcg(ops, b, op, pc)
        if pc == "amg":
            if self.amg_iters0 is None:
                self.amg_iters0 = max(k, 5)
            elif k > 4 * self.amg_iters0 and not rebuild:
                return self.solve(ops, b, setup, jvp_args, rebuild=True)
        self.last_iters = k
        if not np.isfinite(rr) or rr > 1e-3:
            self.mon.log(f"    warning: PCG not converged ({k} it, rel.res {rr:.2e})")
        return x


class StaticSolver:                                                     # solvers.py:481-683
    def __init__(self, model, rtol=5e-3, max_iter=16, linear_solver="auto", tangent="ebe", cg_tol=1e-9,
                 cg_maxiter=20000, verbose=True, monitor=None, line_search=True, graph=True, amg=None,
                 amg_setup="auto", mixed_mode="reliable", operator="gather", async_amg=150000,
                 device_newton=True):
        """``amg``: a prebuilt :class:`linalg.AMG` that every step starts from instead
        of assembling and setting up its own (the serving path keeps one resident
        per mesh); the rebuild rule still applies.  ``device_newton``: run each
        increment (predictor, Newton corrections, line search, linear solves) as one
        graph launch on the device where the configuration allows it (matrix-free
        tangent, mixed solver with reliable updates and graphs, any number of
        blocks); the host loop otherwise."""
        self.m, self.rtol, self.max_iter = model, rtol, max_iter
        self.device_newton = device_newton
        self.mon = monitor or Monitor(verbose)
        self.line_search = line_search
        self.lin = _LinearSystem(model, linear_solver, tangent, cg_tol, cg_maxiter, self.mon, graph, amg_setup,
                                 mixed_mode, operator, async_amg)
        self.lin.pinned_amg = amg
        self.newton_iterations = 0

    def _fields(self, scale=None):
        return dict(scale=scale)

    def _fint(self, u, s, fields):
        return self.m.internal_force(u, s, fields)

    def _ops(self, u, s, fields):
        if self.lin.tangent == "mf":
            self.m.tangent_update(u, s, fields)
            return None
        return self.m.stiffness_ops(u, s, fields)

    def _linsolve(self, u, s, fields, b, setup):
        ops = self._ops(u, s, fields)
        return self.lin.solve(ops, b, setup, (u, s, fields) if ops is None else None)

    # increment control (gfem/solvers.py:525-605): an increment that converges in at
    # most GROW_AFTER Newton corrections lets the next one grow by GROW (capped by the
    # step's dt_max); a failed increment is retried at CUT of its size, and the step
    # fails once that drops below dt_min or the step runs out of increments
    GROW, GROW_AFTER, CUT = 1.5, 5, 0.25

    def _try_increment(self, u, states, t_new, fields, setup, inc):
        """Predictor and Newton iterations of one increment ending at t_new:
        (converged, corrections, u, states); a non-finite residual fails it."""
        fext = setup.fext(t_new)
        start = torch.where(setup.fixed_j, setup.prescribed(t_new), u)
        if self._device_increment_ok():
            return self._device_increment(u, states, start, fext, fields, setup, inc)
        try:
            start = self._predictor(u, states, start, fext, fields, setup)
            ok, its, u_new, s_new, _ = self._newton(start, states, fext, fields, setup, inc)
        except FloatingPointError:
            return False, 0, u, states
        return ok, its, u_new, s_new

    _HOOKS = ("_fint", "_ops", "_linsolve", "_predictor", "_residual", "_newton")

    def _device_increment_ok(self):
        """The increment can run as one device graph: matrix-free tangent, the mixed
        solver with reliable updates and graphs, and none of the host loop's hooks
        replaced by a subclass."""
        lin = self.lin
        return (self.device_newton and lin.method == "mixed" and lin.tangent == "mf"
                and lin.mixed_mode == "reliable" and lin.graph and 1 <= self.max_iter <= 64
                and all(getattr(type(self), h) is getattr(StaticSolver, h) for h in self._HOOKS))

    def _device_increment(self, u, states, start, fext, fields, setup, inc):
        """_predictor + _newton of one increment in one graph launch
        (exfem_newton_increment): the same steps and tests, evaluated on the device."""
        lin = self.lin
        self.m._apply_fields(fields)
        for blk in self.m.blocks:
            blk.set_fixed(setup.fixed)
        if lin.amg is None:                     # the hierarchy the first linear solve would set up
            lin._build_amg(None, setup, (u, states, fields))
        S = lin._solver("mf32", "amg")
        j2 = [blk.material.nstate > 1 for blk in self.m.blocks]
        ok, its, u_new, s_new, self.qref, ratios = S.newton_increment(
            u, [s if f else None for s, f in zip(states, j2)], fext, start, self.qref, self.rtol, self.max_iter,
            self.line_search, lin.cg_tol, lin.cg_maxiter)
        lin.last_iters, lin.last_passes = S.last_iters, S.last_passes
        for it, r in enumerate(ratios, 1):
            self.mon.iteration(inc=inc, it=it, residual=float(r), du=None)
        if not ok:
            return False, its, u, states
        return True, its, u_new, [n if f else s for s, n, f in zip(states, s_new, j2)]

    def solve(self, step, u0=None, states=None, fext0=None, callback=None, state=None, scale=None):
        m = self.m
        st = state or State(m)
        if u0 is not None:
            st.u = torch.as_tensor(u0, dtype=torch.float64, device="cuda")
        if states is not None:
            st.states = states
        if fext0 is not None:
            st.fext = torch.as_tensor(fext0, dtype=torch.float64, device="cuda")
        setup = _Setup(m, step, st)
        self.setup = setup
        self.lin.reset()
        self.qref = 0.0
        fields = self._fields(scale)
        u, states = st.u, st.states
        t, dt = 0.0, min(step.dt_init, step.T)
        history, attempts, total = [], 0, 0
        clock = time.time()
        end = step.T * (1 - 1e-12)
        while t < end and not self.mon.should_stop():
            attempts += 1
            if attempts > step.max_inc:
                raise RuntimeError(f"step {step.name!r}: {step.max_inc} increments used before t reached "
                                   f"{step.T:g} (now {t:.4g})")
            dt = min(dt, step.T - t)
            ok, its, u_new, s_new = self._try_increment(u, states, t + dt, fields, setup, attempts)
            total += its
            self.mon.increment(step=step.name, inc=attempts, t=t + dt if ok else t, dt=dt, iters=its, ok=ok)
            if not ok:
                dt *= self.CUT
                self.mon.log(f"  increment {attempts}: no convergence, retrying with dt {dt:.3g}")
                if dt < step.dt_min:
                    raise RuntimeError(f"step {step.name!r}: increment size {dt:.3g} fell below dt_min "
                                       f"{step.dt_min:g} at t = {t:.4g}")
                continue
            u, states, t = u_new, s_new, t + dt
            history.append((t, its))
            self.mon.log(f"  increment {attempts}: t {t:.4g} (dt {dt:.3g}), {its} Newton corrections, "
                         f"last linear solve {self.lin.last_iters} iterations")
            if callback:
                callback(t, u, states)
            if its <= self.GROW_AFTER:
                dt = min(self.GROW * dt, step.dt_max)
        if t < end:
            self.mon.log(f"  step {step.name!r} stopped at t = {t:.4g} on request")
        self.mon.log(f"  step {step.name!r}: {attempts} increments, {total} Newton corrections, "
                     f"{time.time() - clock:.2f} s")
        fint, _ = self._fint(u, states, fields)
        reactions = (fint - setup.fext(step.T)) * setup.fixed_j
        fe = setup.fext_final()
        st.u, st.states, st.fext = u, states, fe
        st.time += step.T
        st.reactions = reactions
        self.newton_iterations = total
        return u, states, dict(history=history, reactions=reactions, fext=fe, state=st, iterations=total,
                               increments=attempts)

    def _predictor(self, uc, s_old, ut, fext, fields, setup):           # solvers.py:607-624
        delta = ut - uc
        fint, _ = self._fint(uc, s_old, fields)
        if self.lin.tangent == "mf":
            Kd = self.m.tangent_jvp(uc, s_old, delta, fields)
        else:
            ops = self._ops(uc, s_old, fields)
            Kd = self.m.matvec([K for _, K in ops], delta)
        r = setup.free * (fint + Kd - fext)
        rn = float(torch.linalg.norm(r))
        self.qref = max(self.qref, rn)
        if rn == 0.0:
            return ut
        du = self._linsolve(uc, s_old, fields, -r, setup)
        return ut + setup.free * du

    def _residual(self, u, s_old, fext, fields, setup):                # solvers.py:626-630
        fint, s_new = self._fint(u, s_old, fields)
        return setup.free * (fint - fext), fint, s_new

    def _newton(self, u, s_old, fext, fields, setup, inc):              # solvers.py:632-683
        hist = []
        dut = 0.0
        fn_t = float(torch.linalg.norm(fext))
        for it in range(1, self.max_iter + 1):
            r, fint, s_new = self._residual(u, s_old, fext, fields, setup)
            rt = float(torch.linalg.norm(r))
            ft = float(torch.linalg.norm(fint))
            ref = max(fn_t, ft, 1e-3 * self.qref, 1e-30)
            self.qref = max(self.qref, fn_t, ft)
            ratio = rt / ref
            hist.append(ratio)
            self.mon.iteration(inc=inc, it=it, residual=ratio, du=dut)
            if not np.isfinite(rt):
                return False, it, u, s_old, hist
            ut_n = float(torch.linalg.norm(u))
            small_du = dut <= 1e-2 * max(ut_n, 1e-30)
            if ratio <= self.rtol * 1e-2 or (it > 1 and ratio <= self.rtol and small_du):
                return True, it - 1, u, s_new, hist
            du = self._linsolve(u, s_old, fields, -r, setup)
            alpha = 1.0
            if self.line_search:
                rn = rt
                for _ in range(4):
                    ut = u + alpha * du
                    r2 = self._residual(ut, s_old, fext, fields, setup)[0]
                    if float(torch.linalg.norm(r2)) < rn or alpha < 0.2:
                        break
                    alpha *= 0.5
            u = u + alpha * du
            dut = float(torch.linalg.norm(alpha * du))
        return False, self.max_iter, u, s_old, hist
