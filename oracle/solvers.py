"""Oracle: quasi-static Newton procedure of the reference, restated on the CPU.

Test infrastructure only (see ``oracle/__init__.py``).

  * gfem/solvers.py:48-80    ``Step`` (bcs, loads, dloads, dt_init/dt_min/dt_max/max_inc)
  * gfem/solvers.py:104-217  ``_Setup`` for the MPC-free, amplitude-free case used by the
                             hot path: fixed mask, targets ramped from the start state,
                             load groups summed with ``np.add.at``
  * gfem/solvers.py:220-221  ``_ramp``
  * gfem/solvers.py:481-683  ``StaticSolver``: increments with x1.5 growth (<= 5 its) and
                             x0.25 cutback, tangent predictor, Newton with the reference's
                             convergence test and a 4-step backtracking line search
The linear solves use a sparse direct factorisation of the assembled tangent with
fixed DOFs replaced by identity rows (``_LinearSystem.assemble`` + ``linalg.Direct``,
solvers.py:323-326, 417-424), so the oracle's Newton iterates are exact.
"""
import numpy as np
import torch

from . import fem, linalg


class Step:                                                            # solvers.py:48-80
    def __init__(self, name="Step-1", time_period=1.0, dt_init=None, dt_min=None, dt_max=None,
                 max_inc=1000, bcs=(), loads=(), dloads=()):
        self.name, self.T = name, float(time_period)
        self.dt_init = dt_init or self.T
        self.dt_min = dt_min if dt_min is not None else 1e-5 * self.T
        self.dt_max = dt_max or self.T
        self.max_inc = max_inc
        self.bcs, self.loads, self.dloads = list(bcs), list(loads), list(dloads)


def _ramp(t, T):                                                       # solvers.py:220-221
    return min(max(t / T, 0.0), 1.0) if T > 0 else 1.0


class Setup:                                                           # solvers.py:104-217
    def __init__(self, model, step, u_start=None, f_prev=None):
        nd = model.ndof
        self.step = step
        self.fixed = np.zeros(nd, bool)
        self.target = np.zeros(nd)
        for nodes, dof, val in (bc[:3] for bc in step.bcs):
            d = np.asarray(nodes, dtype=np.int64).ravel() * 3 + dof
            self.fixed[d] = True
            self.target[d] = val
        g = np.zeros(nd)
        for nodes, dof, val in (ld[:3] for ld in step.loads):
            np.add.at(g, np.asarray(nodes, dtype=np.int64).ravel() * 3 + dof, val)
        for dl in step.dloads:
            g += np.asarray(dl[0] if isinstance(dl, (tuple, list)) else dl, float)
        self.group = g
        self.fprev = np.zeros(nd) if f_prev is None else np.asarray(f_prev, float)
        self.ustart = np.zeros(nd) if u_start is None else np.asarray(u_start, float)
        self.free = (~self.fixed).astype(float)

    def fext(self, t):
        r = _ramp(t, self.step.T)
        return self.fprev * (1 - r) + self.group * r

    def prescribed(self, t):
        r = _ramp(t, self.step.T)
        tgt = self.ustart + (self.target - self.ustart) * r
        return np.where(self.fixed, tgt, 0.0)


class StaticSolver:                                                    # solvers.py:481-683
    def __init__(self, model, rtol=5e-3, max_iter=16, line_search=True, scale=None, log=None,
                 permc_spec="COLAMD"):
        self.m, self.rtol, self.max_iter = model, rtol, max_iter
        self.permc_spec = permc_spec
        self.line_search = line_search
        self.scale = scale
        self.log = log or (lambda s: None)
        self.linear_solves = 0

    def _fint(self, u, s):
        f, sn = self.m.internal_force(torch.as_tensor(u), s, self.scale)
        return f.numpy(), sn

    def _ops(self, u, s):
        return self.m.stiffness_ops(torch.as_tensor(u), s, self.scale)

    def _linsolve(self, u, s, b, setup):
        ops = [(d, K.numpy()) for d, K in self._ops(u, s)]
        A = linalg.bc_matrix(fem.ops_assemble(ops, self.m.ndof), setup.free)
        self.linear_solves += 1
        return linalg.Direct(A, self.permc_spec).solve(b)

    def solve(self, step, u0=None, states=None):
        m = self.m
        setup = Setup(m, step, u_start=u0)
        self.setup = setup
        u = np.zeros(m.ndof) if u0 is None else np.asarray(u0, float)
        states = m.init_state() if states is None else states
        t, dt, inc, history = 0.0, min(step.dt_init, step.T), 0, []
        self.qref = 0.0
        total = 0
        while t < step.T * (1 - 1e-12):
            inc += 1
            if inc > step.max_inc:
                raise RuntimeError("max increments exceeded")
            dt = min(dt, step.T - t)
            tn = t + dt
            fext = setup.fext(tn)
            ut = np.where(setup.fixed, setup.prescribed(tn), u)
            try:
                ut = self._predictor(u, states, ut, fext, setup)
                ok, it, ui, s_try, rh = self._newton(ut, states, fext, setup)
            except FloatingPointError:
                ok, it, ui, s_try, rh = False, 0, u, states, []
            total += it
            if ok:
                u, states, t = ui, s_try, tn
                history.append((t, it))
                self.log(f"inc {inc} t={t:.4g} dt={dt:.3g} iters={it}")
                if it <= 5:
                    dt = min(dt * 1.5, step.dt_max)
            else:
                dt *= 0.25
                self.log(f"inc {inc} cutback -> dt={dt:.3g}")
                if dt < step.dt_min:
                    raise RuntimeError("time increment smaller than minimum")
        fint, _ = self._fint(u, states)
        reactions = (fint - setup.fext(step.T)) * setup.fixed
        return u, states, dict(history=history, reactions=reactions, iterations=total,
                               increments=inc)

    def _predictor(self, uc, s_old, ut, fext, setup):                  # solvers.py:607-624
        delta = ut - uc
        fint, _ = self._fint(uc, s_old)
        ops = self._ops(uc, s_old)
        Kd = fem.ops_matvec(ops, torch.as_tensor(delta), self.m.ndof).numpy()
        r = setup.free * (fint + Kd - fext)
        self.qref = max(self.qref, float(np.linalg.norm(r)))
        if float(np.linalg.norm(r)) == 0.0:
            return ut
        du = self._linsolve(uc, s_old, -r, setup)
        return ut + setup.free * du

    def _residual(self, u, s_old, fext, setup):                        # solvers.py:626-630
        fint, s_new = self._fint(u, s_old)
        return setup.free * (fint - fext), fint, s_new

    def _newton(self, u, s_old, fext, setup):                          # solvers.py:632-683
        hist = []
        dut = 0.0
        fn_t = float(np.linalg.norm(fext))
        for it in range(1, self.max_iter + 1):
            r, fint, s_new = self._residual(u, s_old, fext, setup)
            rt = float(np.linalg.norm(r))
            ft = float(np.linalg.norm(fint))
            ref = max(fn_t, ft, 1e-3 * self.qref, 1e-30)
            self.qref = max(self.qref, fn_t, ft)
            ratio = rt / ref
            hist.append(ratio)
            if not np.isfinite(rt):
                return False, it, u, s_old, hist
            ut_n = float(np.linalg.norm(u))
            small_du = dut <= 1e-2 * max(ut_n, 1e-30)
            if ratio <= self.rtol * 1e-2 or (it > 1 and ratio <= self.rtol and small_du):
                return True, it - 1, u, s_new, hist
            du = self._linsolve(u, s_old, -r, setup)
            alpha = 1.0
            if self.line_search:
                rn = float(np.linalg.norm(r))
                for _ in range(4):
                    ut = u + alpha * du
                    r2 = self._residual(ut, s_old, fext, setup)[0]
                    if float(np.linalg.norm(r2)) < rn or alpha < 0.2:
                        break
                    alpha *= 0.5
            u = u + alpha * du
            dut = float(np.linalg.norm(alpha * du))
        return False, self.max_iter, u, s_old, hist
