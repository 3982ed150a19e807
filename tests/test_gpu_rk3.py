"""The RK3 short integrators (ATMOS_DYN_tinteg_short_rk3,
scale_atmos_dyn_tinteg_short_rk3.F90:188-576; Heun's "RK3" and "RK3WS2002",
chosen as ATMOS_DYN_Tinteg_short_setup does) against the oracle's
restatement: the short step bit for bit with the HEVI and HEVE stages, the
device entry against the host entry, and the large step with RK3 registered."""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
SHORT_KW = dict(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
                BND_W=False, BND_E=False, BND_S=False, BND_N=False)


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()


def _inputs(g, scheme, short):
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=short == "HEVI")
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    xs = {n: c.state[n].copy(order="F") for n in STATE}
    xs["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xs["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    return a, xs


@pytest.mark.parametrize("tinteg", ["RK3", "RK3WS2002"])
@pytest.mark.parametrize("scheme,short", [("UD3", "HEVI"), ("CD4", "HEVI"), ("UD3KOREN1993", "HEVI"),
                                          ("CD2", "HEVI"), ("UD5", "HEVI"), ("CD6", "HEVI"),
                                          ("CD4", "HEVE"), ("UD5", "HEVE")])
def test_rk3_bit_exact(lib, tinteg, scheme, short):
    g = helpers.small_grid(IMAX=14, JMAX=11, KMAX=18, stretched=True, halo=helpers.halo_of(scheme))
    a, xs = _inputs(g, scheme, short)
    dt = 0.5 if short == "HEVI" else 0.1
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk3(g, scheme, xs, dict(a, dt=dt), ws2002=tinteg == "RK3WS2002", short=short)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.short_type(short)
    lib.tinteg_short_type(tinteg)
    lib.ATMOS_DYN_Tinteg_short_rk3(**a, **xg, **SHORT_KW, dt=dt)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("tinteg", ["RK3", "RK3WS2002"])
def test_rk3_device_entry_matches_host_entry(lib, tinteg):
    import torch

    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20)
    a, xs = _inputs(g, "CD4", "HEVI")
    xh = {n: v.copy(order="F") for n, v in xs.items()}
    lib.setup(g.index_dict(), "CD4", "CD4")
    lib.tinteg_short_type(tinteg)
    lib.ATMOS_DYN_Tinteg_short_rk3(**a, **xh, **SHORT_KW, dt=0.5)

    def dev(x):
        return torch.from_numpy(np.ravel(x, order="K").copy()).cuda() if isinstance(x, np.ndarray) and x.ndim >= 2 else x

    ad = {k: dev(v) for k, v in a.items()}
    xd = {k: dev(v) for k, v in xs.items()}
    lib.ATMOS_DYN_Tinteg_short_rk3_dev(**ad, **xd, **SHORT_KW, dt=0.5)
    lib.check()
    for n, v in xh.items():
        got = xd[n].cpu().numpy().reshape(v.shape, order="F")
        assert np.array_equal(got, v), n


@pytest.mark.parametrize("tinteg", ["RK3", "RK3WS2002"])
@pytest.mark.parametrize("case", ["dry", "moist_fct"])
def test_large_step_rk3_parity(lib, tinteg, case):
    from test_gpu_parity import _field_err, _run_large_both

    c = mkinit.config(1, scale=0.3) if case == "dry" else mkinit.config(2, scale=0.04)
    st_ref, st_gpu = _run_large_both(c, 2, lib, tinteg=tinteg)
    for n in STATE:
        err = _field_err(st_gpu[n], st_ref[n], c.g)
        assert err <= 1e-10, f"{n}: {err:.3e}"
    for iq in range(c.QA):
        err = _field_err(st_gpu["QTRC"][..., iq], st_ref["QTRC"][..., iq], c.g)
        assert err <= 1e-10, f"QTRC[{iq}]: {err:.3e}"


def test_rk3_needs_registration(lib):
    g = helpers.small_grid()
    a, xs = _inputs(g, "UD3", "HEVI")
    lib.setup(g.index_dict(), "UD3", "UD3")
    with pytest.raises(hevi.HeviError, match="RK4") as e:
        lib.ATMOS_DYN_Tinteg_short_rk3(**a, **xs, **SHORT_KW, dt=0.5)
    assert e.value.code == 5
    with pytest.raises(hevi.HeviError, match="RK3WS2002"):
        lib.tinteg_short_type("RK2")
