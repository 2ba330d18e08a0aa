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


def fit_trust_region(loglik_grad, theta0, lb, ub, max_iter=60, gtol=1e-3, delta0=0.5, delta_max=1.0, log=None,
                     state=None, ftol=0.0):
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
    the free coordinates is at most gtol, when two accepted steps in a row
    raise f by less than ftol (an objective whose values carry noise of that
    size cannot resolve more), when the radius falls below 1e-8, or after
    max_iter iterations.  Returns (theta, f, evaluations,
    history) with one (theta, f) pair per accepted step.  state (a dict, may
    be None): state["B"], when present, is the initial Hessian model in phi,
    and receives the final one; state["stop"] receives the stop reason
    ("gtol", "stall", "radius" or "max_iter"), state["gphi"] the final
    gradient in phi and state["updates"] the number of BFGS updates."""
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
    first_update = True
    stalls = 0
    updates = 0
    if state is not None and state.get("B") is not None:
        B = np.array(state["B"], dtype=np.float64)
        first_update = False
    delta = delta0
    history = [(th.copy(), f)]

    def projected(gp, ph):
        free = ~(((ph <= plo + 1e-12) & (gp < 0)) | ((ph >= phi_hi - 1e-12) & (gp > 0)))
        return np.max(np.abs(gp[free])) if np.any(free) else 0.0

    stop = "max_iter"
    for it in range(max_iter):
        if projected(gphi, phi) <= gtol:
            stop = "gtol"
            break
        if delta < 1e-8:
            stop = "radius"
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
                if first_update:
                    # the scaled identity of the first step is replaced by
                    # the curvature seen along it (y.y / s.y, Shanno-Phua)
                    B = np.eye(n) * ((y @ y) / sy)
                    first_update = False
                Bs = B @ s
                B = B - np.outer(Bs, Bs) / (s @ Bs) + np.outer(y, y) / sy
                updates += 1
        if rho > 1.25 and np.linalg.norm(d) < 0.8 * delta:
            # an interior step that gained more than the model promised: the
            # model is too curved along it (the flat ridge); halve it so the
            # next steps grow geometrically instead of crawling
            B = 0.5 * B
        if rho >= 0.1:
            small = 0.0 <= fc - f < ftol
            phi, f, gphi = cand_phi, fc, gc
            history.append((np.exp(phi), f))
            stalls = stalls + 1 if small else 0
            if stalls >= 2:
                stop = "stall"
                break
            if rho > 0.75 and np.linalg.norm(d) > 0.8 * delta:
                delta = min(2.0 * delta, delta_max)
        else:
            delta = 0.25 * min(delta, np.linalg.norm(d))
        if rho < 0.25 and rho >= 0.1:
            delta *= 0.5
        if log:
            log("trust region %d: theta %s f %.12g rho %.3g delta %.3g |g_phi| %.3g" % (
                it, list(np.exp(phi)), f, rho, delta, projected(gphi, phi)))
    if projected(gphi, phi) <= gtol:
        stop = "gtol"
    if state is not None:
        state["B"] = B
        state["gphi"] = gphi
        state["stop"] = stop
        state["updates"] = updates
    return np.exp(phi), f, evals, history


def start_point(loglik, z, lb, ub, nbeta=7):
    """A start for the gradient drivers: sigma^2 = the sample variance of z,
    nu = 1/2 (both clipped to the box), and the range beta that maximises
    loglik over nbeta values spaced geometrically across [lb, ub] (nbeta
    evaluations; a failing one counts as -inf).  Returns (theta, evaluations)."""
    lb = np.asarray(lb, dtype=np.float64)
    ub = np.asarray(ub, dtype=np.float64)
    th = np.clip(np.array([float(np.var(z)), np.sqrt(lb[1] * ub[1]), 0.5] + list(lb[3:])), lb, ub)
    best, fbest = th.copy(), -np.inf
    for b in np.geomspace(lb[1], ub[1], nbeta):
        t = th.copy()
        t[1] = b
        try:
            fv = loglik(t)
        except Exception:
            fv = -np.inf
        if np.isfinite(fv) and fv > fbest:
            best, fbest = t, fv
    return best, nbeta


def value_newton_polish(loglik, theta, B, lb, ub, signal=1e-2, rounds=2):
    """Newton steps on a quadratic model fitted to values of the objective
    only (in phi = log theta), for an objective whose gradient is less
    accurate than its values -- the INT8-sliced path, whose log-likelihood is
    good to ~1e-9 relative but whose adjoint gradient is good to ~1e-4 of
    its largest entry.  The model is fitted in the eigenbasis u_i of the
    Hessian model B, with steps h_i = sqrt(2 signal / |lambda_i|) so that every
    sampled change of f is about `signal` (far above the values' noise):
    f at the centre, at +- h_i u_i and at h_i u_i + h_j u_j (10 values for
    three parameters) give the gradient, the diagonal and the cross
    curvatures exactly for a quadratic.  The Newton step of that model (at
    most 3 h_i along each direction, inside the box) is taken when it raises
    f.  Returns (theta, f(theta), evaluations)."""
    lo, hi = np.log(np.asarray(lb, dtype=np.float64)), np.log(np.asarray(ub, dtype=np.float64))
    phi = np.log(np.asarray(theta, dtype=np.float64))
    w, V = np.linalg.eigh(np.asarray(B, dtype=np.float64))
    n = phi.size

    def f(p):
        try:
            v = loglik(np.exp(np.clip(p, lo, hi)))
        except Exception:
            return -np.inf
        return v if np.isfinite(v) else -np.inf

    f0 = f(phi)
    evals = 1
    for _ in range(rounds):
        h = np.sqrt(2.0 * signal / np.maximum(np.abs(w), 1e-12))
        h = np.minimum(h, 0.5)
        D = V * h  # columns: the scaled sample directions
        fp = np.array([f(phi + D[:, i]) for i in range(n)])
        fm = np.array([f(phi - D[:, i]) for i in range(n)])
        evals += 2 * n
        g = (fp - fm) / 2.0
        H = np.diag(fp - 2.0 * f0 + fm)
        for i in range(n):
            for j in range(i + 1, n):
                fij = f(phi + D[:, i] + D[:, j])
                evals += 1
                H[i, j] = H[j, i] = fij - f0 - g[i] - g[j] - 0.5 * (H[i, i] + H[j, j])
        if not (np.all(np.isfinite(H)) and np.all(np.isfinite(g))):
            break
        ev = np.linalg.eigvalsh(H)
        if ev.max() >= 0.0:
            break  # not concave at this scale: keep the point
        x = np.clip(np.linalg.solve(H, -g), -3.0, 3.0)
        cand = np.clip(phi + D @ x, lo, hi)
        fc = f(cand)
        evals += 1
        if not fc > f0:
            break
        phi, f0 = cand, fc
        if np.max(np.abs(x)) < 0.1:
            break
    return np.exp(phi), f0, evals


def _newton_step_size(state):
    """max |d log theta| of the Newton step -B^-1 g of the trust region's
    final model; inf when the model is singular or has seen fewer BFGS
    updates than twice the parameters (a model that has not learned the flat
    ridge misjudges the step along it)."""
    if state.get("updates", 0) < 2 * len(state.get("gphi", ())):
        return np.inf
    try:
        return float(np.max(np.abs(np.linalg.solve(state["B"], state["gphi"]))))
    except (np.linalg.LinAlgError, KeyError, TypeError):
        return np.inf


def fit_mixed(session, lb, ub, theta0=None, gtol=0.1, ftol=1e-4, log=None, newton_tol=5e-4):
    """Mixed-precision adjoint-gradient MLE, entirely on the INT8-sliced
    objective (precision 3): a start from start_point (unless theta0 is
    given), the trust-region maximiser driven by the sliced adjoint gradient
    (stopping at gtol / ftol, the noise level of that gradient), then
    value_newton_polish with sliced log-likelihood values -- skipped when the
    gradient itself reached gtol and the Newton step of the trust region's
    model (learned over at least 2 n BFGS updates) would move log theta by
    at most newton_tol: along a flat ridge a gradient at its noise level can
    still leave theta 1e-3 away.  Leaves the session in
    FP64.  Returns (theta_hat, loglik, sliced evaluations (log-likelihood and
    gradient), sliced log-likelihood-only evaluations, theta after the
    gradient stage)."""
    session.set_sliced()
    z = session.z()
    if theta0 is None:
        start, ne = start_point(lambda t: session.loglik(t), z, lb, ub)
    else:
        start, ne = np.asarray(theta0, dtype=np.float64), 0
    st = {}
    th1, f1, ev1, _ = fit_trust_region(lambda t: session.loglik(t, grad=True), start, lb, ub, gtol=gtol, ftol=ftol,
                                       log=log, state=st)
    if log:
        log("sliced gradient stage: %d evaluations, theta %s, loglik %.12g" % (ev1, list(th1), f1))
    if st["stop"] == "gtol" and _newton_step_size(st) <= newton_tol:
        # the sliced gradient reached the optimum to its noise level and the
        # model's Newton step from there moves theta by less than newton_tol
        th, f, ne2 = th1, f1, 0
    else:
        th, f, ne2 = value_newton_polish(lambda t: session.loglik(t), th1, st["B"], lb, ub)
    if log:
        log("sliced value-based Newton polish (%s stop): %d evaluations, theta %s, loglik %.12g" % (
            st["stop"], ne2, list(th), f))
    session.set_fp64()
    return th, f, ev1, ne + ne2, th1


def fit_fp64(session, lb, ub, theta0=None, gtol=1e-3, ftol=1e-7, log=None):
    """The same gradient driver in plain FP64 (start_point with FP64 values,
    the trust region on the FP64 adjoint gradient).  Returns (theta_hat,
    loglik, gradient evaluations, log-likelihood-only evaluations)."""
    session.set_fp64()
    z = session.z()
    if theta0 is None:
        start, ne = start_point(lambda t: session.loglik(t), z, lb, ub)
    else:
        start, ne = np.asarray(theta0, dtype=np.float64), 0
    th, f, ev, _ = fit_trust_region(lambda t: session.loglik(t, grad=True), start, lb, ub, gtol=gtol, ftol=ftol,
                                    log=log)
    return th, f, ev, ne
