"""The differentiated short step: the pass form the tangent-linear and adjoint
linearise reproduces the fused forward step; the tangent-linear model agrees
with central finite differences of the forward; the adjoint is its transpose
(dot-product test); and the gradient of the warm-bubble cost J through many
steps with checkpointing matches central finite differences along random
directions."""
import numpy as np
import pytest

from scale_b200 import adjoint, hevi, mkinit

pytestmark = pytest.mark.gpu


def _case(scheme="UD3", I=24, J=20, K=20):
    c = mkinit.ensemble_member(I, J, K, 3)
    if scheme != "UD3":
        c.scheme = scheme
    return c


@pytest.fixture(params=["UD3", "CD4"])
def model(request):
    c = _case(request.param)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        yield adjoint.Model(c)
    finally:
        hevi.finalize()


def test_pass_form_reproduces_fused_step(model):
    X = model.state()
    model.boundary(X)
    Xa, Xb = X.clone(), X.clone()
    for _ in range(3):
        model.step(Xa)
        model.step_passes(Xb)
    hevi.check()
    d = (Xa - Xb).abs().max().item()
    assert d <= 1e-12 * Xa.abs().max().item(), d


# UD3 takes the upwind stencil by the sign of the face velocity, so the
# discrete model has kinks where a face velocity is zero; a finite
# perturbation that crosses one leaves a first-order error in the central
# difference (measured 1e-6..3e-4 for eps = 1e-8..1e-5 on this case, falling
# with eps), while CD4 is smooth and agrees to round-off.
FD_TOL = {"CD4": 1e-7, "UD3": 1e-3}


def test_tangent_linear_matches_finite_differences(model):
    import torch

    X = model.state()
    model.boundary(X)
    for _ in range(5):  # away from the rest state, where the upwind switches sit at zero velocity
        model.step(X)
    rng = np.random.default_rng(1)
    dx = torch.from_numpy(rng.standard_normal(X.numel())).cuda()
    dx *= X.abs()  # relative perturbation
    model.boundary(dx)
    X1, dX = X.clone(), dx.clone()
    for _ in range(3):
        model.tlm(X1, dX)
    eps = 1e-7
    Xp, Xm = X + eps * dx, X - eps * dx
    for _ in range(3):
        model.step(Xp)
        model.step(Xm)
    fd = (Xp - Xm) / (2 * eps)
    hevi.check()
    e = (fd - dX).abs() / dX.abs().max()
    err = e.max().item()
    med = e.median().item()
    print(f"{model.case.scheme}: tangent-linear vs central difference, max relative error {err:.3e}, median {med:.3e}")
    assert err < FD_TOL[model.case.scheme], err
    # away from the cells a switch crossing reaches, UD3 agrees as CD4 does
    assert med < 1e-8, med


@pytest.mark.parametrize("scheme", ["UD3KOREN1993", "CD2"])
def test_adjoint_dot_product_other_schemes(scheme):
    c = _case(scheme)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        m = adjoint.Model(c)
        X = m.state()
        m.boundary(X)
        for _ in range(3):
            m.step(X)
        r = adjoint.dot_product_test(m, X, 2)
        assert r["rel_diff"] < 1e-11, r
        # the pass form reproduces the fused step for this scheme as well
        Xa, Xb = X.clone(), X.clone()
        m.step(Xa)
        m.step_passes(Xb)
        hevi.check()
        assert (Xa - Xb).abs().max().item() <= 1e-12 * Xa.abs().max().item()
    finally:
        hevi.finalize()


def test_adjoint_dot_product(model):
    X = model.state()
    model.boundary(X)
    r = adjoint.dot_product_test(model, X, 3)
    assert r["rel_diff"] < 1e-11, r


@pytest.mark.parametrize("scheme", ["CD4", "UD3"])
def test_gradient_against_finite_differences_with_checkpoints(scheme):
    c = _case(scheme, 24, 24, 20)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        # cost box scaled to the 12 km x 12 km x 5 km test domain
        p = adjoint.Problem(c, nsteps=12, K=4, box=((3e3, 9e3), (3e3, 9e3), (1e3, 3e3)), spinup=5)
        r = adjoint.gradient_check(p, ndirs=4, eps=1e-6)
        print(scheme, "gradient vs central differences:", [f"{row['rel_err']:.2e}" for row in r["directions"]])
        assert r["max_rel_err"] < (1e-6 if scheme == "CD4" else 1e-4), r
        # the same gradient with every state stored (K = nsteps) and K = 1; the
        # adjoint passes add with atomics, so sums may differ in the last bits
        g4 = p.value_and_grad()[1]
        p.K = 12
        g12 = p.value_and_grad()[1]
        p.K = 1
        g1 = p.value_and_grad()[1]
        for a, b, c_ in zip(g4, g12, g1):
            scale = a.abs().max().item()
            assert (a - b).abs().max().item() <= 1e-12 * scale
            assert (a - c_).abs().max().item() <= 1e-12 * scale
    finally:
        hevi.finalize()


def test_double_double_step_agrees_with_the_pass_form(model):
    """The double-double step (hi + lo) rounds to the FP64 pass-form step: the
    two differ by the FP64 model's own rounding, far below 1e-10 of each field."""
    import torch

    X = model.state()
    model.boundary(X)
    hi, lo = X.clone(), torch.zeros_like(X)
    Y = X.clone()
    for _ in range(3):
        model.step_passes(Y)
        model.step_dd(hi, lo)
    hevi.check()
    n = model.n3
    for q in range(5):
        a, b = Y[q * n:(q + 1) * n], hi[q * n:(q + 1) * n] + lo[q * n:(q + 1) * n]
        scale = max(b.abs().max().item(), 1e-300)
        assert (a - b).abs().max().item() <= 1e-10 * scale, q
        # the lo parts are small next to the hi parts
        assert lo[q * n:(q + 1) * n].abs().max().item() <= 1e-15 * scale, q


def test_gradient_against_double_double_differences():
    """With both perturbed runs in double-double arithmetic the central
    difference at eps = 1e-6 carries no FP64 rounding of the forward model:
    the adjoint gradient (CD4) agrees with it to 1e-6."""
    c = _case("CD4", 24, 24, 20)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        p = adjoint.Problem(c, nsteps=12, K=4, box=((3e3, 9e3), (3e3, 9e3), (1e3, 3e3)), spinup=5)
        r = adjoint.gradient_check(p, ndirs=4, eps=1e-6, dd=True)
        print("gradient vs double-double central differences:", [f"{row['rel_err']:.2e}" for row in r["directions"]])
        assert r["max_rel_err"] < 1e-6, r
    finally:
        hevi.finalize()
