"""Maximum-likelihood drivers on top of the library's objectives.

`fit_two_stage` is the reduced-precision MLE: the reference driver's
derivative-free maximiser (start at the lower bounds,
examples/examples.c:263-264) on the INT8-sliced objective to a loose
tolerance, then `newton_polish` in FP64 from its end point.  The polish is a bounded Newton
iteration in log-parameters with the adjoint gradient, a Hessian from
central differences of gradients at the start and BFGS updates after; near
the optimum of the flat sigma^2-beta ridge of the Matern likelihood it
converges in a few steps where a quasi-Newton or a derivative-free method
keeps crawling along the ridge.
"""
from __future__ import annotations

import numpy as np


def newton_polish(loglik_grad, theta, lb, ub, max_steps=8, rel_h=1e-4, xtol=1e-6):
    """Refines a maximiser of f on the box [lb, ub] (lb > 0).

    loglik_grad(theta) -> (f, grad).  The iteration runs in phi = log theta,
    where the sigma^2-beta ridge of the Matern likelihood is nearly straight.
    The Hessian in phi is formed once by central differences of gradients
    (2 n gradient evaluations) and then carried by BFGS updates; each step is
    the Newton step d = -H^-1 g_phi when it is an ascent direction (else a
    short gradient step), projected onto the box and halved until f does not
    decrease.  A failing evaluation (an exception, or a non-finite value)
    counts as f = -inf: it rejects a trial step, and at the start point it
    ends the polish.  Stops when the accepted relative step is below xtol,
    after max_steps, or when no step improves f.  Returns (theta, f, gradient
    evaluations)."""
    lb = np.asarray(lb, dtype=np.float64)
    ub = np.asarray(ub, dtype=np.float64)
    th = np.clip(np.asarray(theta, dtype=np.float64), lb, ub)
    n = th.size

    def fg(t):
        """f and gradient; an evaluation that fails (e.g. a covariance that is
        not positive definite) counts as f = -inf."""
        try:
            fv, gv = loglik_grad(t)
        except Exception:
            return -np.inf, np.full(n, np.nan)
        gv = np.asarray(gv, dtype=np.float64)
        return (fv, gv) if np.isfinite(fv) and np.all(np.isfinite(gv)) else (-np.inf, np.full(n, np.nan))

    f, g = fg(th)
    evals = 1
    if not np.isfinite(f):
        return th, f, evals
    phi = np.log(th)
    gphi = g * th
    H = np.empty((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = rel_h
        tp, tm = np.exp(phi + e), np.exp(phi - e)
        _, gp = fg(tp)
        _, gm = fg(tm)
        evals += 2
        H[:, j] = (gp * tp - gm * tm) / (2 * rel_h)
    H = 0.5 * (H + H.T)
    if not np.all(np.isfinite(H)):
        H = -np.eye(n) * max(np.max(np.abs(gphi)), 1.0)
    for _ in range(max_steps):
        try:
            d = np.linalg.solve(H, -gphi)
        except np.linalg.LinAlgError:
            d = None
        if d is None or not np.all(np.isfinite(d)) or gphi @ d <= 0.0:
            d = 1e-2 * gphi / max(np.max(np.abs(gphi)), 1e-300)
        t = 1.0
        accepted = False
        step = 0.0
        while t >= 1.0 / 64:
            cand = np.clip(np.exp(phi + t * d), lb, ub)
            fc, gc = fg(cand)
            evals += 1
            if np.isfinite(fc) and fc >= f:
                step = np.max(np.abs(cand - th) / th)
                phi_new = np.log(cand)
                gphi_new = np.asarray(gc, dtype=np.float64) * cand
                # BFGS update of the (negative definite) Hessian of f in phi
                sv, yv = phi_new - phi, gphi_new - gphi
                sy = sv @ yv
                if sy < 0.0:
                    Hs = H @ sv
                    H = H - np.outer(Hs, Hs) / (sv @ Hs) + np.outer(yv, yv) / sy
                th, f, g, phi, gphi = cand, fc, np.asarray(gc, dtype=np.float64), phi_new, gphi_new
                accepted = True
                break
            t *= 0.5
        if not accepted or step < xtol:
            break
    return th, f, evals


def fit_two_stage(session, lb, ub, ftol_abs=1e-3, maxeval=400, polish_steps=8, log=None):
    """Reduced-precision MLE: the derivative-free maximiser on the sliced
    objective (precision 3) to a loose tolerance (two accepted steps in a row
    that change loglik by less than ftol_abs, or maxeval evaluations), then
    the FP64 Newton polish, which does the fine convergence along the ridge.
    Leaves the session in FP64.  log(msg), when given, receives progress.
    Returns (theta_hat, loglik, sliced evaluations, FP64 gradient evaluations,
    theta after the first stage)."""
    session.set_sliced()
    th1, f1, ev1 = session.fit_bobyqa(lb, ub, ftol_abs=ftol_abs, maxeval=maxeval)
    if log:
        log("stage 1 (sliced, derivative-free): %d evaluations, theta %s, loglik %.10g" % (ev1, list(th1), f1))
    session.set_fp64()
    th, f, ev2 = newton_polish(lambda t: session.loglik(t, grad=True), th1, lb, ub, max_steps=polish_steps)
    if log:
        log("stage 2 (FP64 Newton): %d gradient evaluations, theta %s, loglik %.12g" % (ev2, list(th), f))
    return th, f, ev1, ev2, th1
