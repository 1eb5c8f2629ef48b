"""Ice fit: maximum-likelihood per-layer scattering and absorption coefficients from
per-(event, DOM) charges, by L-BFGS on the adjoint gradient.

No counterpart in the reference's propagator; llh/DirectFit fits ice parameters with
repeated forward runs and finite differences (llh/llh.cxx:1435-1634).  Here every
evaluation is one recording forward pass over all events plus the replay of the detected
photons (PPC.gradient), so an iteration costs about one forward pass instead of 2 x 342.

The parameters are log scale factors u (be_j = be0_j exp(u_be_j), ba_j = ba0_j exp(u_ba_j)),
bounded to |u| <= log(bound); the objective is -LL.  Per-photon random streams keep the
objective's random numbers fixed from one evaluation to the next.

The objective (plus the optional smoothness / ridge penalty) is a Monte Carlo estimate: its
value moves in small jumps as hits appear and disappear, while the gradient estimates the
derivative of its expectation.  A line search
that insists on the Wolfe conditions spends many evaluations chasing those jumps, so the
L-BFGS direction (two-loop recursion, Nocedal & Wright, Numerical Optimization, alg. 7.4)
is taken inside a trust region on max |du| instead: a step that lowers the objective is
kept and the region grows; one that raises it is undone and the region shrinks."""
import time

import numpy as np


def lbfgs_direction(g, S, Y):
    """-H g for the L-BFGS inverse-Hessian estimate H built from the pairs (s, y)."""
    q = g.copy()
    stack = []
    for s, y in zip(reversed(S), reversed(Y)):
        rho = 1.0 / float(y @ s)
        a = rho * float(s @ q)
        q -= a * y
        stack.append((a, rho, s, y))
    if S:
        q *= float(S[-1] @ Y[-1]) / float(Y[-1] @ Y[-1])
    for a, rho, s, y in reversed(stack):
        b = rho * float(y @ q)
        q += s * (a - b)
    return -q


def minimize_trust_lbfgs(fg, x0, iters, lo, hi, radius=0.05, max_radius=0.3, memory=10, callback=None):
    """Minimises f with gradient from fg(x) -> (f, g) within the box [lo, hi]."""
    x = np.array(x0, np.float64)
    f, g = fg(x)
    S, Y = [], []
    evals, accepted = 1, 0
    for _ in range(iters):
        d = lbfgs_direction(g, S, Y) if S else -g
        if float(d @ g) >= 0:  # not a descent direction: restart from steepest descent
            S.clear()
            Y.clear()
            d = -g
        step = d * min(1.0, radius / max(np.abs(d).max(), 1e-300))
        xn = np.clip(x + step, lo, hi)
        fn, gn = fg(xn)
        evals += 1
        s, y = xn - x, gn - g
        if float(s @ y) > 1e-12 * np.linalg.norm(s) * np.linalg.norm(y):
            S.append(s)
            Y.append(y)
            if len(S) > memory:
                S.pop(0)
                Y.pop(0)
        if fn < f:
            x, f, g = xn, fn, gn
            accepted += 1
            radius = min(max_radius, radius * 1.5)
        else:
            radius *= 0.5
        if callback:
            callback(x, f)
    return x, f, evals, accepted


def penalty(u, n, smooth, ridge):
    """(smooth/2) sum (u_j+1 - u_j)^2 + (ridge/2) sum u_j^2 over each block of n layers, and
    its gradient."""
    p, g = 0.0, np.zeros_like(u)
    for k in range(len(u) // n):
        v = u[k * n:(k + 1) * n]
        dv = np.diff(v)
        p += 0.5 * smooth * float(dv @ dv) + 0.5 * ridge * float(v @ v)
        gv = ridge * v
        gv[:-1] -= smooth * dv
        gv[1:] += smooth * dv
        g[k * n:(k + 1) * n] = gv
    return p, g


def fit_ice(ctx, bunches, observed, events, be0=None, ba0=None, iters=20, fit=("be", "ba"), bound=2.0,
            hit_cap=None, radius=0.05, smooth=0.0, ridge=0.0, callback=None, graph=True):
    """ctx: an initialised PPC (after ini()).  observed: (events, gsize) charges, the event of
    a bunch being its q.  Layers are 10 m thick while a flasher's light samples the ice over
    tens of metres, so neighbouring layers trade off against each other; `smooth` and `ridge`
    add a penalty on layer-to-layer differences and on the distance from the starting ice
    (in units of log-likelihood per unit of log scale squared).  With `graph` each evaluation
    is one replay of a CUDA graph holding the forward pass and the adjoint
    (PPC.gradient_graph); otherwise PPC.gradient runs them eagerly.  Returns the fitted be,
    ba, the LL of every evaluation and timings."""
    if be0 is None or ba0 is None:
        b, a = ctx.get_ice()
        be0 = b if be0 is None else be0
        ba0 = a if ba0 is None else ba0
    be0 = np.asarray(be0, np.float64)
    ba0 = np.asarray(ba0, np.float64)
    n = len(be0)
    use_be, use_ba = "be" in fit, "ba" in fit
    nx = n * (use_be + use_ba)
    hist = []

    def unpack(u):
        ube = u[:n] if use_be else np.zeros(n)
        uba = u[n * use_be:n * use_be + n] if use_ba else np.zeros(n)
        return be0 * np.exp(ube), ba0 * np.exp(uba)

    G = ctx.gradient_graph(bunches, observed, events=events, hit_cap=hit_cap) if graph else None

    def fg(u):
        be, ba = unpack(u)
        t0 = time.perf_counter()
        if G is not None:
            r = G.run(be.astype(np.float32), ba.astype(np.float32), counts=False)
        else:
            ctx.set_ice(be.astype(np.float32), ba.astype(np.float32))
            r = ctx.gradient(bunches, observed=observed, events=events, hit_cap=hit_cap)
        dt = time.perf_counter() - t0
        g = []
        if use_be:
            g.append(r["g_be"] * be)
        if use_ba:
            g.append(r["g_ba"] * ba)
        hist.append({"ll": r["ll"], "seconds": dt, "forward_ms": r["info"]["forward_ms"],
                     "backward_ms": r["info"]["backward_ms"]})
        if callback:
            callback(len(hist), r["ll"], be, ba)
        p, gp = penalty(u, n, smooth, ridge)
        return -r["ll"] + p, -np.concatenate(g) + gp

    lim = np.log(bound)
    t0 = time.perf_counter()
    u, f, evals, accepted = minimize_trust_lbfgs(fg, np.zeros(nx), iters, -lim, lim, radius=radius)
    f -= penalty(u, n, smooth, ridge)[0]  # the likelihood part: -LL
    wall = time.perf_counter() - t0
    be, ba = unpack(u)
    ctx.set_ice(be.astype(np.float32), ba.astype(np.float32))
    if G is not None:
        G.close()
    return {"be": be, "ba": ba, "ll": -f, "history": hist, "iterations": iters, "evaluations": evals,
            "accepted": accepted, "seconds": wall, "seconds_per_iteration": wall / max(1, iters)}
