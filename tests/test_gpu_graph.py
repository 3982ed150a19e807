"""The short-step sequence (numerical filter, RK4 and the boundary/halo
update) recorded once as a CUDA graph and replayed: the replayed steps give the
same state bit for bit as the same number of eager calls, and the kernel-launch
count grows by the recorded launches per replay."""
import numpy as np
import pytest

from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


def _device_problem(c):
    import torch

    g = c.g
    N3 = int(np.prod(g.shape))
    RT2P, DPRES0, REF_rhot = mkinit.large_prep(c)
    dev = lambda x: torch.from_numpy(np.ravel(x, order="K").copy()).cuda()  # noqa: E731
    z = lambda k=1: torch.zeros(k * N3, dtype=torch.float64, device="cuda")  # noqa: E731
    X = {n: dev(c.state[n]) for n in STATE}
    ref = {n: dev(v) for n, v in c.ref.items()}
    b = dict(mflx=z(3), tflx=z(3), nd=z(15), tend={n: z() for n in ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")},
             ref=ref, dp0=dev(DPRES0), rt2p=dev(RT2P), refr=dev(REF_rhot),
             GS=torch.ones(7 * N3, dtype=torch.float64, device="cuda"),
             J0=torch.zeros(7 * N3, dtype=torch.float64, device="cuda"),
             MAPF=torch.ones(g.IA * g.JA * 8, dtype=torch.float64, device="cuda"),
             cor=torch.zeros(g.IA * g.JA, dtype=torch.float64, device="cuda"))
    return X, b


def _short_step(c, X, b):
    g = c.g
    grid = dict(CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ,
                RFDX=g.RFDX, RFDY=g.RFDY)
    hevi.ATMOS_DYN_numfilter_coef_dev(num_diff=b["nd"], CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX,
                                      FDY=g.FDY, DT=c.dt, REF_dens=b["ref"]["REF_dens"],
                                      REF_pott=b["ref"]["REF_pott"], ND_COEF=c.nd_coef, ND_ORDER=1,
                                      ND_SFC_FACT=1.0, ND_USE_RS=True, **X)
    hevi.ATMOS_DYN_Tinteg_short_rk4_dev(
        PROG=None, mflx_hi=b["mflx"], tflx_hi=b["tflx"], DPRES0=b["dp0"], RT2P=b["rt2p"], CORIOLI=b["cor"],
        num_diff=b["nd"], wdamp_coef=np.zeros(g.KA), divdmp_coef=0.0, DDIV=None, FLAG_FCT_MOMENTUM=False,
        FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True, PHI=b["ref"]["PHI"], GSQRT=b["GS"], J13G=b["J0"],
        J23G=b["J0"], J33G=1.0, MAPF=b["MAPF"], REF_dens=b["ref"]["REF_dens"], REF_rhot=b["refr"], BND_W=False,
        BND_E=False, BND_S=False, BND_N=False, dt=c.dt, **X, **b["tend"], **grid)
    hevi.boundary_dev(**X)


def _host(c, X):
    return {n: X[n].cpu().numpy().reshape(c.g.shape, order="F") for n in STATE}


@pytest.mark.parametrize("cfg", [1, 2])
def test_graph_replay_matches_eager_steps(cfg):
    nsteps = 6
    c = mkinit.config(cfg, scale=1 / 8) if cfg == 2 else mkinit.config(cfg)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        X, b = _device_problem(c)
        for _ in range(nsteps):
            _short_step(c, X, b)
        hevi.check()
        eager = _host(c, X)
    finally:
        hevi.finalize()

    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        X, b = _device_problem(c)
        _short_step(c, X, b)  # eager warm-up: one-time checks and table uploads
        l0 = hevi.kernel_launches()
        _short_step(c, X, b)
        per_step = hevi.kernel_launches() - l0
        hevi.capture_begin()
        _short_step(c, X, b)  # recorded, not run
        hevi.capture_end()
        l1 = hevi.kernel_launches()
        assert l1 == l0 + per_step
        hevi.replay(nsteps - 2)
        assert hevi.kernel_launches() == l1 + (nsteps - 2) * per_step
        hevi.check()
        graphed = _host(c, X)
    finally:
        hevi.finalize()
    for n in STATE:
        assert np.array_equal(graphed[n], eager[n]), n


def test_capture_rejects_nesting_and_empty_replay():
    c = mkinit.config(1)
    hevi.setup(c.g.index_dict(), c.scheme, c.scheme_tracer)
    try:
        with pytest.raises(hevi.HeviError):
            hevi.replay(1)
        with pytest.raises(hevi.HeviError):
            hevi.capture_end()
        hevi.capture_begin()
        with pytest.raises(hevi.HeviError):
            hevi.capture_begin()
        hevi.capture_end()  # an empty graph
        hevi.replay(1)
        hevi.check()
    finally:
        hevi.finalize()
