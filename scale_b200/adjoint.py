"""Differentiation of the HEVI short step: the forward/adjoint C-ABI pair as
torch.autograd Functions, with checkpoint-and-recompute over many steps, and
the gradient-check harness (central finite differences, tangent-linear
dot-product test).

The model is the one the library differentiates (scale_hevi_adjoint_setup):
short steps of a single flat-terrain domain with the large-step quantities
(DPRES0, RT2P, REF_rhot) fixed and zero tendencies, as a run of short steps
from one large-step preparation (scale_atmos_dyn_tstep_large_fvm_heve.F90:
428-470, 847-944). A state is one device tensor of 5*KA*IA*JA doubles: DENS,
MOMZ, MOMX, MOMY, RHOT in the reference's (KA,IA,JA) layout. The product
kernels do all the work; torch only holds the buffers and the autograd graph.
"""
from __future__ import annotations

import numpy as np

from . import hevi, mkinit

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


class Model:
    """Parameters of the differentiated short step for a mkinit.Case, on the
    library's device (the library must be set up for the case's grid)."""

    def __init__(self, case):
        import torch

        g = case.g
        self.case, self.g = case, g
        self.n3 = int(np.prod(g.shape))
        RT2P, DPRES0, REF_rhot = mkinit.large_prep(case)
        dev = lambda x: torch.from_numpy(np.ravel(x, order="F").copy()).cuda()  # noqa: E731
        self.par = dict(DPRES0=dev(DPRES0), RT2P=dev(RT2P), REF_rhot=dev(REF_rhot), REF_dens=dev(case.ref["REF_dens"]),
                        REF_pott=dev(case.ref["REF_pott"]), PHI=dev(case.ref["PHI"]),
                        CORIOLI=torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda"))
        hevi.call("scale_hevi_adjoint_setup", **self.par, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX,
                  FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY,
                  wdamp_coef=np.zeros(g.KA), dt=case.dt, ND_COEF=case.nd_coef, ND_SFC_FACT=1.0, J33G=1.0)

    def state(self):
        """The case's initial state as one (5*N3) device tensor."""
        import torch

        return torch.cat([torch.from_numpy(np.ravel(self.case.state[n], order="F").copy()) for n in STATE]).cuda()

    # ---- the C-ABI pair (in place on device tensors) ----
    def step(self, X) -> None:
        hevi.call("scale_hevi_short_step_dev", X=X)

    def step_passes(self, X) -> None:
        hevi.call("scale_hevi_short_step_passes_dev", X=X)

    def tlm(self, X, dX) -> None:
        hevi.call("scale_hevi_short_step_tlm_dev", X=X, dX=dX)

    def step_dd(self, X_hi, X_lo) -> None:
        """One step in double-double arithmetic; the state is X_hi + X_lo."""
        hevi.call("scale_hevi_short_step_dd_dev", X_hi=X_hi, X_lo=X_lo)

    def adjoint(self, X, lam) -> None:
        hevi.call("scale_hevi_short_step_adjoint_dev", X=X, lam=lam)

    def boundary(self, X) -> None:
        n = self.n3
        hevi.boundary_dev(*(X[q * n:(q + 1) * n] for q in range(5)))

    def boundary_adjoint(self, lam) -> None:
        hevi.call("scale_hevi_boundary_adjoint_dev", lam=lam)


def _autograd():
    import torch

    class BoundaryFill(torch.autograd.Function):
        """Vertical boundary values and periodic halo of a state."""

        @staticmethod
        def forward(ctx, X, model):
            ctx.model = model
            Y = X.detach().clone()
            model.boundary(Y)
            return Y

        @staticmethod
        def backward(ctx, gY):
            lam = gY.detach().clone().contiguous()
            ctx.model.boundary_adjoint(lam)
            return lam, None

    class ShortSteps(torch.autograd.Function):
        """nsteps short steps; the backward pass keeps one state every K steps
        and recomputes the K states of a segment before running its adjoint
        steps in reverse."""

        @staticmethod
        def forward(ctx, X0, model, nsteps, K):
            ctx.model, ctx.nsteps, ctx.K = model, nsteps, K
            X = X0.detach().clone()
            ckpt = []
            for s in range(nsteps):
                if s % K == 0:
                    ckpt.append(X.clone())
                model.step(X)
            ctx.ckpt = ckpt
            return X

        @staticmethod
        def backward(ctx, gX):
            model, nsteps, K = ctx.model, ctx.nsteps, ctx.K
            lam = gX.detach().clone().contiguous()
            for seg in range(len(ctx.ckpt) - 1, -1, -1):
                s0 = seg * K
                n = min(K, nsteps - s0)
                states = [ctx.ckpt[seg].clone()]
                for _ in range(n - 1):
                    X = states[-1].clone()
                    model.step(X)
                    states.append(X)
                for X in reversed(states):
                    model.adjoint(X, lam)
            ctx.ckpt = None
            return lam, None, None, None

    return BoundaryFill, ShortSteps


def cost_box(case, x_range=(20e3, 44e3), y_range=(20e3, 44e3), z_range=(2e3, 6e3)):
    """Mask (KA,IA,JA) of the interior cells whose centres lie in the box and
    their volumes CDZ*CDX*CDY."""
    g = case.g
    zc, xc, yc = g.CZ, g.CX, g.CY
    inside = lambda c, r: (c >= r[0]) & (c <= r[1])  # noqa: E731
    m = inside(zc, z_range)[:, None, None] & inside(xc, x_range)[None, :, None] & inside(yc, y_range)[None, None, :]
    interior = np.zeros(g.shape, dtype=bool)
    interior[g.KS - 1:g.KE, g.IS - 1:g.IE, g.JS - 1:g.JE] = True
    vol = g.CDZ[:, None, None] * g.CDX[None, :, None] * g.CDY[None, None, :]
    return m & interior, vol


class Problem:
    """J(theta0, MOMX0, MOMY0) = 1/2 sum over the box of (theta - theta_base)^2
    vol after nsteps short steps, where the initial state has the DENS and
    MOMZ of the start state, RHOT = DENS * theta0, and the boundary fill
    applied. The start state is the case's state after `spinup` short steps:
    from rest every velocity is exactly zero, where the UD3 upwind switches of
    the discrete model have no derivative."""

    def __init__(self, case, nsteps: int, K: int, box=None, spinup: int = 0):
        import torch

        self.case, self.nsteps, self.K = case, nsteps, K
        self.model = Model(case)
        self.BoundaryFill, self.ShortSteps = _autograd()
        g = case.g
        mask, vol = cost_box(case, *(box or ()))
        n3 = self.model.n3
        f = lambda a: torch.from_numpy(np.ravel(a, order="F").copy()).cuda()  # noqa: E731
        self.w = f(np.where(mask, vol, 0.0))
        self.theta_base = f(case.ref["REF_pott"])
        X = self.model.state()
        self.model.boundary(X)
        for _ in range(spinup):
            self.model.step(X)
        hevi.check()
        self.DENS0, self.MOMZ0 = X[:n3].clone(), X[n3:2 * n3].clone()
        self.MOMX0, self.MOMY0 = X[2 * n3:3 * n3].clone(), X[3 * n3:4 * n3].clone()
        self.theta0 = X[4 * n3:] / X[:n3]
        self.n3, self.g = n3, g

    def J(self, theta0, MOMX0, MOMY0):
        import torch

        X0 = torch.cat([self.DENS0, self.MOMZ0, MOMX0, MOMY0, self.DENS0 * theta0])
        X0 = self.BoundaryFill.apply(X0, self.model)
        X = self.ShortSteps.apply(X0, self.model, self.nsteps, self.K)
        n = self.n3
        th = X[4 * n:] / X[:n]
        d = th - self.theta_base
        return 0.5 * torch.sum(d * d * self.w)

    def value_and_grad(self):
        th = self.theta0.clone().requires_grad_(True)
        u = self.MOMX0.clone().requires_grad_(True)
        v = self.MOMY0.clone().requires_grad_(True)
        J = self.J(th, u, v)
        J.backward()
        return float(J.detach()), (th.grad, u.grad, v.grad)

    def J_of(self, d, eps):
        import torch

        with torch.no_grad():
            return float(self.J(self.theta0 + eps * d[0], self.MOMX0 + eps * d[1], self.MOMY0 + eps * d[2]))

    def theta_of(self, d, eps):
        """Potential temperature after the steps from the state perturbed by eps*d."""
        import torch

        with torch.no_grad():
            th0, u, v = self.theta0 + eps * d[0], self.MOMX0 + eps * d[1], self.MOMY0 + eps * d[2]
            X0 = torch.cat([self.DENS0, self.MOMZ0, u, v, self.DENS0 * th0])
            X0 = self.BoundaryFill.apply(X0, self.model)
            X = self.ShortSteps.apply(X0, self.model, self.nsteps, self.K)
            n = self.n3
            return X[4 * n:] / X[:n]

    def theta_of_dd(self, d, eps):
        """theta_of in double-double arithmetic (scale_hevi_short_step_dd_dev):
        the perturbed start state is formed exactly, every step rounds at about
        1e-32, and theta = RHOT/DENS comes back as a (hi, lo) pair of numpy arrays."""
        import torch

        n = self.n3
        host = lambda t: t.detach().cpu().numpy()  # noqa: E731
        D0, W0 = host(self.DENS0), host(self.MOMZ0)
        th_h, th_l = _two_sum(host(self.theta0), host(eps * d[0]))
        u_h, u_l = _two_sum(host(self.MOMX0), host(eps * d[1]))
        v_h, v_l = _two_sum(host(self.MOMY0), host(eps * d[2]))
        r_h, r_l = dd_mul(D0, 0.0 * D0, th_h, th_l)
        z = np.zeros_like(D0)
        hi = torch.from_numpy(np.concatenate([D0, W0, u_h, v_h, r_h])).cuda()
        lo = torch.from_numpy(np.concatenate([z, z, u_l, v_l, r_l])).cuda()
        self.model.boundary(hi)
        self.model.boundary(lo)
        for _ in range(self.nsteps):
            self.model.step_dd(hi, lo)
        hevi.check()
        h, l = host(hi), host(lo)
        with np.errstate(divide="ignore", invalid="ignore"):
            return dd_div(h[4 * n:], l[4 * n:], h[:n], l[:n])

    def J_diff_dd(self, d, eps):
        """J_diff with both runs in double-double arithmetic: the difference of
        the two trajectories then carries no rounding of the forward model (FP64
        leaves about 1e-16 of theta per operation, which divided by 2 eps sets a
        floor of 1e-6..1e-5 on the finite difference at eps = 1e-6)."""
        tph, tpl = self.theta_of_dd(d, eps)
        tmh, tml = self.theta_of_dd(d, -eps)
        dh, dl = dd_add(tph, tpl, -tmh, -tml)
        diff = dh + dl
        base = self.theta_base.cpu().numpy()
        w = self.w.cpu().numpy()
        m = w > 0.0
        terms = diff[m] * (((tph[m] - base[m]) + tpl[m]) + ((tmh[m] - base[m]) + tml[m])) * w[m]
        return 0.5 * float(np.sum(terms))

    def J_diff(self, d, eps):
        """J(X + eps d) - J(X - eps d), differenced cell by cell before the sum:
        a^2 - b^2 = (a - b)(a + b) with a, b the deviations from the base state of
        the two runs. J itself (about 2.5e10 on the warm bubble) would leave a
        rounding floor of about 1e-16 J in the difference of the two totals."""
        import torch

        with torch.no_grad():
            tp, tm = self.theta_of(d, eps), self.theta_of(d, -eps)
            return float(0.5 * torch.sum((tp - tm) * ((tp - self.theta_base) + (tm - self.theta_base)) * self.w))


# ---- double-double arithmetic on the host (error-free transforms in numpy's
# IEEE float64: Knuth's two-sum, Veltkamp's split and Dekker's product) ----
def _fast_sum(a, b):
    s = a + b
    return s, b - (s - a)


def _two_sum(a, b):
    s = a + b
    v = s - a
    return s, (a - (s - v)) + (b - v)


def _split(a):
    c = 134217729.0 * a  # 2^27 + 1
    hi = c - (c - a)
    return hi, a - hi


def _two_prod(a, b):
    p = a * b
    ah, al = _split(a)
    bh, bl = _split(b)
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


def dd_add(ah, al, bh, bl):
    s, e = _two_sum(ah, bh)
    t, f = _two_sum(al, bl)
    s, e = _fast_sum(s, e + t)
    return _fast_sum(s, e + f)


def dd_mul(ah, al, bh, bl):
    p, e = _two_prod(ah, bh)
    return _fast_sum(p, e + (ah * bl + al * bh))


def dd_div(ah, al, bh, bl):
    q1 = ah / bh
    rh, rl = dd_add(ah, al, *(-x for x in dd_mul(bh, bl, q1, 0.0 * q1)))
    q2 = rh / bh
    rh, rl = dd_add(rh, rl, *(-x for x in dd_mul(bh, bl, q2, 0.0 * q2)))
    q3 = rh / bh
    s, e = _fast_sum(q1, q2)
    return dd_add(s, e, q3, 0.0 * q3)


def interior_direction(g, rng, device="cuda"):
    """A random perturbation of (theta0, MOMX0, MOMY0) on the interior cells,
    scaled to 1 K and 1 kg m-2 s-1 at most."""
    import torch

    out = []
    for scale in (1.0, 1.0, 1.0):
        a = np.zeros(g.shape)
        a[g.KS - 1:g.KE, g.IS - 1:g.IE, g.JS - 1:g.JE] = rng.uniform(-scale, scale, (g.KMAX, g.IMAX, g.JMAX))
        out.append(torch.from_numpy(np.ravel(a, order="F").copy()).to(device))
    return out


def gradient_check(problem: Problem, ndirs: int = 8, eps=1e-6, seed: int = 0, dd: bool = False) -> dict:
    """Adjoint gradient against central finite differences along ndirs
    seeded random directions: relative error |FD - <grad, d>| / |FD| for each
    step size in eps (a number or a sequence); max_rel_err is over the first.
    dd: the finite differences from double-double forward runs (J_diff_dd)."""
    eps_list = [eps] if np.isscalar(eps) else list(eps)
    J0, grad = problem.value_and_grad()
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(ndirs):
        d = interior_direction(problem.g, rng)
        ad = float(sum((gq * dq).sum() for gq, dq in zip(grad, d)))
        row = {"adjoint": ad}
        for e in eps_list:
            fd = (problem.J_diff_dd(d, e) if dd else problem.J_diff(d, e)) / (2 * e)
            row[f"fd_{e:g}"] = fd
            row[f"rel_err_{e:g}"] = abs(fd - ad) / max(abs(fd), 1e-300)
        row["rel_err"] = row[f"rel_err_{eps_list[0]:g}"]
        rows.append(row)
    return {"J": J0, "eps": eps_list, "directions": rows, "max_rel_err": max(r["rel_err"] for r in rows)}


def dot_product_test(model: Model, X0, nsteps: int, seed: int = 0) -> dict:
    """<M' dx, w> against <dx, M'^T w> for nsteps short steps (tangent-linear
    run forward, adjoint run backward over the stored states)."""
    import torch

    g = model.g
    rng = np.random.default_rng(seed)
    n3 = model.n3
    dx = torch.from_numpy(rng.standard_normal(5 * n3)).cuda()
    w = torch.from_numpy(rng.standard_normal(5 * n3)).cuda()
    # perturb interior-only quantities consistently: fill the boundary of dx
    model.boundary(dx)
    X = X0.clone()
    states = []
    dX = dx.clone()
    for _ in range(nsteps):
        states.append(X.clone())
        model.tlm(X, dX)
    lam = w.clone()
    for Xs in reversed(states):
        model.adjoint(Xs, lam)
    lhs = float((dX * w).sum())
    rhs = float((dx * lam).sum())
    hevi.check()
    return {"tl_dot_w": lhs, "dx_dot_adj": rhs, "rel_diff": abs(lhs - rhs) / max(abs(lhs), 1e-300)}
