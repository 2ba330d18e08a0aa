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


def _tr_step(g, B, delta, lo, hi):
    """Maximiser of the quadratic model g.d + d.B d / 2 (B negative definite)
    in the ball |d| <= delta, then clipped to the box lo <= d <= hi."""
    n = g.size
    try:
        d = np.linalg.solve(B, -g)
    except np.linalg.LinAlgError:
        d = None
    if d is None or not np.all(np.isfinite(d)) or g @ d <= 0.0 or np.linalg.norm(d) > delta:
        # (B - mu I) d = -g with mu >= 0 chosen so that |d| = delta (bisection in mu)
        lam_max = float(np.max(np.linalg.eigvalsh(B)))
        mu_lo = max(0.0, lam_max + 1e-12 * max(1.0, abs(lam_max)))
        mu_hi = mu_lo + np.linalg.norm(g) / delta + 1.0
        for _ in range(100):
            mu = 0.5 * (mu_lo + mu_hi)
            d = np.linalg.solve(B - mu * np.eye(n), -g)
            if np.linalg.norm(d) > delta:
                mu_lo = mu
            else:
                mu_hi = mu
        d = np.linalg.solve(B - mu_hi * np.eye(n), -g)
    return np.clip(d, lo, hi)


def fit_trust_region(loglik_grad, theta0, lb, ub, max_iter=60, gtol=1e-3, delta0=0.5, delta_max=2.0, log=None,
                     state=None):
    """Gradient-based maximiser of f on the box [lb, ub] (lb > 0), for an
    objective whose value and adjoint gradient come from one call
    (loglik_grad(theta) -> (f, grad)).

    It works in phi = log theta with a trust region: each step maximises the
    quadratic model (gradient, BFGS Hessian) inside a ball of radius delta in
    phi, clipped to the box; a step is accepted when f rises by at least a
    tenth of the model's prediction.  A failing evaluation (an exception, a
    non-finite value: e.g. a covariance that is not positive definite in the
    working precision) rejects the step and shrinks the region, so the
    iteration never leaves the region where the objective is defined -- the
    large-range corner of the Matern box, where Sigma is numerically singular,
    is approached only as far as the likelihood rises.  The radius starts at
    delta0 and never exceeds delta_max (a factor e^2 per step).

    Stops when the scaled projected gradient max_k |d f / d log theta_k| over
    the free coordinates is at most gtol, or when the radius falls below
    1e-8, or after max_iter iterations.  Returns (theta, f, evaluations,
    history) with one (theta, f) pair per accepted step.  state (a dict, may
    be None): state["B"], when present, is the initial Hessian model in phi,
    and receives the final one."""
    lb = np.asarray(lb, dtype=np.float64)
    ub = np.asarray(ub, dtype=np.float64)
    th = np.clip(np.asarray(theta0, dtype=np.float64), lb, ub)
    n = th.size
    plo, phi_hi = np.log(lb), np.log(ub)

    def fg(t):
        try:
            fv, gv = loglik_grad(t)
        except Exception:
            return -np.inf, None
        gv = np.asarray(gv, dtype=np.float64)
        if not (np.isfinite(fv) and np.all(np.isfinite(gv))):
            return -np.inf, None
        return fv, gv * t  # gradient in phi

    phi = np.log(th)
    f, gphi = fg(th)
    evals = 1
    if not np.isfinite(f):
        raise RuntimeError("the objective fails at the start point %s" % list(th))
    B = -np.eye(n) * max(np.max(np.abs(gphi)) / delta0, 1.0)
    if state is not None and state.get("B") is not None:
        B = np.array(state["B"], dtype=np.float64)
    delta = delta0
    history = [(th.copy(), f)]

    def projected(gp, ph):
        free = ~(((ph <= plo + 1e-12) & (gp < 0)) | ((ph >= phi_hi - 1e-12) & (gp > 0)))
        return np.max(np.abs(gp[free])) if np.any(free) else 0.0

    for it in range(max_iter):
        if projected(gphi, phi) <= gtol or delta < 1e-8:
            break
        d = _tr_step(gphi, B, delta, plo - phi, phi_hi - phi)
        pred = gphi @ d + 0.5 * d @ B @ d
        if pred <= 0.0 or np.linalg.norm(d) == 0.0:
            B = -np.eye(n) * max(np.max(np.abs(gphi)) / delta, 1.0)
            delta *= 0.25
            continue
        cand_phi = phi + d
        fc, gc = fg(np.exp(cand_phi))
        evals += 1
        rho = (fc - f) / pred if np.isfinite(fc) else -np.inf
        if gc is not None:
            s, y = d, gc - gphi
            sy = s @ y
            if sy < -1e-12 * np.linalg.norm(s) * np.linalg.norm(y):
                Bs = B @ s
                B = B - np.outer(Bs, Bs) / (s @ Bs) + np.outer(y, y) / sy
        if rho >= 0.1:
            phi, f, gphi = cand_phi, fc, gc
            history.append((np.exp(phi), f))
            if rho > 0.75 and np.linalg.norm(d) > 0.8 * delta:
                delta = min(2.0 * delta, delta_max)
        else:
            delta = 0.25 * min(delta, np.linalg.norm(d))
        if rho < 0.25 and rho >= 0.1:
            delta *= 0.5
        if log:
            log("trust region %d: theta %s f %.12g rho %.3g delta %.3g |g_phi| %.3g" % (
                it, list(np.exp(phi)), f, rho, delta, projected(gphi, phi)))
    if state is not None:
        state["B"] = B
        state["gphi"] = gphi
    return np.exp(phi), f, evals, history


def fit_mixed(session, lb, ub, theta0=None, gtol=1e-2, polish_gtol=1e-3, polish_iter=0, log=None):
    """Mixed-precision adjoint-gradient MLE: the trust-region maximiser on the
    INT8-sliced objective and its sliced adjoint gradient (precision 3) from
    theta0 (default: the lower bounds, where the reference's driver starts,
    examples/examples.c:263-264), then, when polish_iter > 0, at most
    polish_iter FP64 gradient steps from its end point that reuse the sliced
    run's Hessian model.  Leaves the session in FP64.  Returns (theta_hat,
    loglik, sliced evaluations, FP64 evaluations, theta after the sliced
    stage)."""
    start = np.asarray(lb if theta0 is None else theta0, dtype=np.float64)
    session.set_sliced()
    st = {}
    th1, f1, ev1, _ = fit_trust_region(lambda t: session.loglik(t, grad=True), start, lb, ub, gtol=gtol, log=log,
                                       state=st)
    if log:
        log("sliced stage: %d evaluations, theta %s, loglik %.12g" % (ev1, list(th1), f1))
    session.set_fp64()
    if polish_iter <= 0:
        return th1, f1, ev1, 0, th1
    th, f, ev2, _ = fit_trust_region(lambda t: session.loglik(t, grad=True), th1, lb, ub, max_iter=polish_iter,
                                     gtol=polish_gtol, delta0=0.05, log=log, state=st)
    if log:
        log("FP64 polish: %d evaluations, theta %s, loglik %.12g" % (ev2, list(th), f))
    return th, f, ev1, ev2, th1
