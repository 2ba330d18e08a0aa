"""Gradient-based MLE on top of the C ABI.

``MaternLogLikelihood`` is a ``torch.autograd.Function`` whose forward calls
``exageostat_b200_loglik`` with a gradient buffer (the adjoint path of the
library: alpha = Sigma^-1 z, Sigma^-1 from the factor, dSigma/dtheta generated
on the fly) and whose backward returns that gradient, so the GPU log-likelihood
composes with torch code and can be checked with ``torch.autograd.gradcheck``
against finite differences.

``fit_lbfgsb`` maximises the log-likelihood with scipy's L-BFGS-B using the
same gradient, beside the derivative-free ``Session.fit_bobyqa``.
"""
from __future__ import annotations

import numpy as np
import torch


class MaternLogLikelihood(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta: torch.Tensor, session) -> torch.Tensor:
        th = theta.detach().to("cpu", torch.float64).numpy()
        ll, g = session.loglik(th, grad=True)
        ctx.save_for_backward(torch.from_numpy(np.asarray(g, dtype=np.float64)))
        return torch.tensor(ll, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None


def loglik(theta: torch.Tensor, session) -> torch.Tensor:
    return MaternLogLikelihood.apply(theta, session)


def fit_lbfgsb(session, lb, ub, x0=None, ftol=1e-12, gtol=1e-6, maxiter=500):
    """Maximise the log-likelihood over the box [lb, ub] with L-BFGS-B and the
    library's gradient.  Returns (theta_hat, loglik, evaluations)."""
    from scipy.optimize import minimize

    lb = np.asarray(lb, dtype=np.float64)
    ub = np.asarray(ub, dtype=np.float64)
    x0 = 0.5 * (lb + ub) if x0 is None else np.asarray(x0, dtype=np.float64)
    count = [0]

    def fun(t):
        count[0] += 1
        ll, g = session.loglik(t, grad=True)
        if not np.isfinite(ll):
            return 1e300, np.zeros_like(t)
        return -ll, -np.asarray(g)

    r = minimize(fun, x0, jac=True, bounds=list(zip(lb, ub)), method="L-BFGS-B",
                 options={"ftol": ftol, "gtol": gtol, "maxiter": maxiter})
    return r.x, -r.fun, count[0]
