"""The host-array large step (ATMOS_DYN_Tstep_large_fvm_heve) copies its inputs
in on a second stream and each group of outputs back as soon as it is final,
overlapping the copies with the kernels. Its results must be those of the
device-array entry on the same inputs, bit for bit, for every output
(scale_atmos_dyn_tstep_large_fvm_heve.F90 intent(inout)/(out) arguments: the
state, QTRC, mflx_hi, tflx_hi, num_diff), with pinned host buffers (truly
asynchronous copies) as well as with pageable ones."""
import numpy as np
import pytest

import oracle
from scale_b200 import hevi, mkinit

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
OUTS = (("mflx_hi", (3,)), ("tflx_hi", (3,)), ("num_diff", (5, 3)))


@pytest.fixture
def lib(gpu):
    yield hevi
    hevi.finalize()


def _pinned_like(a):
    import torch

    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    v = t.numpy().reshape(a.shape, order="F")
    v[...] = a
    return t, v


def _common(c):
    g = c.g
    tp = {n: g.zeros() for n in ("DENS_tp", "MOMZ_tp", "MOMX_tp", "MOMY_tp", "RHOT_tp")}
    rng = np.random.default_rng(7)
    for v in tp.values():  # small physics tendencies, so that every input group matters
        v[...] = 1e-6 * rng.standard_normal(v.shape)
    rhoq = g.zeros(c.QA) if c.QA else None
    if c.QA:
        rhoq[...] = 1e-9 * rng.standard_normal(rhoq.shape)
    cor = np.full((g.IA, g.JA), 1e-4, order="F")
    aq = mkinit.aq_props(c.QA) if c.QA else (None, None, None, None)
    kw = dict(QA=c.QA, CORIOLI=cor, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, RCDZ=g.RCDZ,
              RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ, RFDX=g.RFDX, RFDY=g.RFDY, J33G=1.0, AQ_R=aq[0], AQ_CV=aq[1],
              AQ_CP=aq[2], AQ_MASS=aq[3], ND_COEF=c.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=True,
              wdamp_coef=np.zeros(g.KA), divdmp_coef=0.05, FLAG_FCT_TRACER=c.fct, FLAG_FCT_ALONG_STREAM=True,
              DTLS=c.dtl, DTSS=c.dt)
    return tp, rhoq, kw


def _host(c, nlarge, pinned):
    g = c.g
    tp, rhoq, kw = _common(c)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)
    keep = []

    def H(a):
        if a is None or not pinned:
            return None if a is None else a.copy(order="F")
        t, v = _pinned_like(a)
        keep.append(t)
        return v

    st = {n: H(c.state[n]) for n in STATE}
    q = H(c.state["QTRC"]) if c.QA else None
    out = {n: H(g.zeros(*s)) for n, s in OUTS}
    ref = {n: H(v) for n, v in c.ref.items()}
    kw["CORIOLI"] = H(kw["CORIOLI"])
    tph = {n: H(v) for n, v in tp.items()}
    hevi.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    for _ in range(nlarge):
        hevi.ATMOS_DYN_Tstep_large_fvm_heve(
            QTRC=q, RHOQ_tp=H(rhoq), PHI=ref["PHI"], GSQRT=GS, J13G=J13, J23G=J23, MAPF=MAPF,
            REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"], REF_pres=ref["REF_pres"], **st, **out, **tph, **kw)
    res = {n: np.array(v, order="F") for n, v in {**st, **out}.items()}
    if c.QA:
        res["QTRC"] = np.array(q, order="F")
    hevi.finalize()
    return res


def _device(c, nlarge):
    import torch

    g = c.g
    tp, rhoq, kw = _common(c)
    GS, J13, J23, MAPF = oracle.flat_metrics(g)

    def D(a):
        return None if a is None else torch.from_numpy(np.ravel(a, order="K").copy()).cuda()

    st = {n: D(c.state[n]) for n in STATE}
    q = D(c.state["QTRC"]) if c.QA else None
    out = {n: D(g.zeros(*s)) for n, s in OUTS}
    ref = {n: D(v) for n, v in c.ref.items()}
    kw["CORIOLI"] = D(kw["CORIOLI"])
    hevi.setup(g.index_dict(), c.scheme, c.scheme_tracer)
    for _ in range(nlarge):
        hevi.ATMOS_DYN_Tstep_large_fvm_heve_dev(
            QTRC=q, RHOQ_tp=D(rhoq), PHI=ref["PHI"], GSQRT=D(GS), J13G=D(J13), J23G=D(J23), MAPF=D(MAPF),
            REF_dens=ref["REF_dens"], REF_pott=ref["REF_pott"], REF_pres=ref["REF_pres"], **st, **out,
            **{n: D(v) for n, v in tp.items()}, **kw)
    hevi.check()
    torch.cuda.synchronize()

    def back(t, shape):
        return t.cpu().numpy().reshape(shape, order="F")

    res = {n: back(st[n], g.shape) for n in STATE}
    res.update({n: back(out[n], g.shape + s) for n, s in OUTS})
    if c.QA:
        res["QTRC"] = back(q, g.shape + (c.QA,))
    hevi.finalize()
    return res


def _same(a, b):
    assert a.keys() == b.keys()
    for n in a:
        x, y = a[n], b[n]
        assert x.shape == y.shape, n
        assert np.array_equal(x, y, equal_nan=True), f"{n}: max diff {np.nanmax(np.abs(x - y)):.3e}"


@pytest.mark.parametrize("case", ["dry", "moist_fct"])
def test_host_entry_matches_device_entry(lib, case):
    c = mkinit.config(1, scale=0.3) if case == "dry" else mkinit.config(2, scale=0.04)
    dev = _device(c, 2)
    _same(_host(c, 2, pinned=True), dev)
    _same(_host(c, 2, pinned=False), dev)
    assert all(np.isfinite(dev[n]).all() for n in STATE)
