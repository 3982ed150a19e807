"""Edge sizes, bit for bit against the oracle:
- the smallest domains the setup accepts: KMAX = 4 (5 for UD5/CD6) and
  IMAX = JMAX = IHALO;
- the largest column, KMAX = 256 (KA = 260, the column arrays of the stage
  kernel at their maximum);
- ragged tiles: several 16-column tiles with a partial last one, and columns
  whose last 32-level chunk holds a single level.
The stage kernel, the RK4 short step, the numerical filter and the FCT tracer
step run through the C-ABI; the oracle computes the same call on the CPU."""
import numpy as np
import pytest

import helpers
import oracle

pytestmark = pytest.mark.gpu

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")

# (IMAX, JMAX, KMAX, scheme, stretched)
SIZES = [
    (2, 2, 4, "UD3", False),
    (2, 3, 4, "CD4", True),
    (3, 3, 5, "UD5", True),
    (3, 4, 5, "CD6", False),
    (5, 37, 256, "CD4", False),
    (40, 3, 33, "UD3KOREN1993", False),
    (33, 2, 64, "CD2", True),
    (19, 18, 97, "UD5", True),
]


@pytest.fixture
def lib(gpu):
    from scale_b200 import hevi

    yield hevi
    hevi.finalize()


def _grid(IMAX, JMAX, KMAX, scheme, stretched):
    return helpers.small_grid(IMAX=IMAX, JMAX=JMAX, KMAX=KMAX, DX=300.0, DY=300.0, DZ=1000.0 / KMAX * 8,
                              stretched=stretched, halo=helpers.halo_of(scheme))


def _stage_kw(a, o):
    kw = dict(a)
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    return kw


@pytest.mark.parametrize("size", SIZES, ids=lambda s: "x".join(map(str, s[:3])) + "-" + s[3])
def test_stage_edge_sizes(lib, size):
    g = _grid(*size)
    scheme = size[3]
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, dtrk=0.5, full=True)
    o_ref = helpers.stage_outputs(g)
    oracle.tstep_short(g, scheme, o_ref, a)
    o_gpu = helpers.stage_outputs(g)
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_short_fvm_hevi(**_stage_kw(a, o_gpu))
    for n in o_ref:
        assert helpers.same(o_gpu[n], o_ref[n]), f"{n}: max rel diff {helpers.max_rel(o_gpu[n], o_ref[n]):.3e}"


@pytest.mark.parametrize("size", [SIZES[0], SIZES[2], SIZES[4]], ids=lambda s: "x".join(map(str, s[:3])) + "-" + s[3])
def test_rk4_edge_sizes(lib, size):
    g = _grid(*size)
    scheme = size[3]
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    a = helpers.short_inputs(c, full=True)
    for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
        a.pop(k)
    xs = {n: c.state[n].copy(order="F") for n in STATE}
    xs["mflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xs["tflx_hi"] = np.full(g.shape + (3,), 7.0, order="F")
    xg = {n: v.copy(order="F") for n, v in xs.items()}
    oracle.tinteg_short_rk4(g, scheme, xs, dict(a, dt=0.5))
    lib.setup(g.index_dict(), scheme, scheme)
    kw = dict(a, **xg)
    kw.update(PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True,
              BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=0.5)
    lib.ATMOS_DYN_Tinteg_short_rk4(**kw)
    for n in xs:
        assert helpers.same(xg[n], xs[n]), f"{n}: max rel diff {helpers.max_rel(xg[n], xs[n]):.3e}"


@pytest.mark.parametrize("size,order", [(SIZES[0], 1), ((2, 2, 6, "UD3", False), 2), (SIZES[2], 1), (SIZES[4], 2)],
                         ids=["2x2x4-o1", "2x2x6-o2", "3x3x5-halo3", "5x37x256-o2"])
def test_numfilter_edge_sizes(lib, size, order):
    g = _grid(*size)
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    ref_nd = g.zeros(5, 3)
    oracle.numfilter(g, ref_nd, c.state, c.ref, DT=0.5, ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7)
    got = np.full(g.shape + (5, 3), np.nan, order="F")
    lib.setup(g.index_dict(), "UD3", "UD3")
    lib.ATMOS_DYN_numfilter_coef(num_diff=got, DENS=c.state["DENS"], MOMZ=c.state["MOMZ"], MOMX=c.state["MOMX"],
                                 MOMY=c.state["MOMY"], RHOT=c.state["RHOT"], CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY,
                                 FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5, REF_dens=c.ref["REF_dens"],
                                 REF_pott=c.ref["REF_pott"], ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7,
                                 ND_USE_RS=True)
    for v in range(5):
        for d in range(3):
            assert helpers.same(got[..., v, d], ref_nd[..., v, d]), f"num_diff(:,:,:,{v+1},{d+1})"


@pytest.mark.parametrize("size", SIZES, ids=lambda s: "x".join(map(str, s[:3])) + "-" + s[3])
def test_fct_tracer_edge_sizes(lib, size):
    # even KA takes the fused limiter (one strip and tile shorter than its
    # 16 rows, 8 columns and 32 levels, or many of them), odd KA the three-kernel form
    from test_gpu_parity import _tracer_inputs

    g = _grid(*size)
    scheme = size[3]
    c = helpers.small_case(g)
    helpers.perturb_state(c)
    q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
    ref = np.full(g.shape, np.nan, order="F")
    oracle.tstep_tracer(g, scheme, ref, q, q0, rhoq, d0, d, mflx, g.zeros(3), GS, MAPF, 2.5, True, True)
    got = np.full(g.shape, np.nan, order="F")
    lib.setup(g.index_dict(), scheme, scheme)
    lib.ATMOS_DYN_Tstep_tracer_fvm_heve(QTRCo=got, QTRC=q, QTRC0=q0, RHOQ_t=rhoq, DENS0=d0, DENS=d, mflx_hi=mflx,
                                        num_diff=g.zeros(3), GSQRT=GS, MAPF=MAPF, CDZ=g.CDZ, RCDZ=g.RCDZ,
                                        RCDX=g.RCDX, RCDY=g.RCDY, dtl=2.5, FLAG_FCT_TRACER=True,
                                        FLAG_FCT_ALONG_STREAM=True)
    assert helpers.same(got, ref), f"max rel diff {helpers.max_rel(got, ref):.3e}"


def test_higher_order_filter_rejects_short_columns(lib):
    """calc_diff3 (scale_atmos_dyn_common.F90:1695-1696) mirrors levels KS+2 and
    KS+3 of the w-point quantity before it has written them when KMAX < 6; the
    higher-order filter reads those levels, so it is refused there."""
    from scale_b200 import hevi

    g = _grid(2, 2, 5, "UD3", False)
    c = helpers.small_case(g)
    lib.setup(g.index_dict(), "UD3", "UD3")
    with pytest.raises(hevi.HeviError, match="KMAX >= 6") as e:
        lib.ATMOS_DYN_numfilter_coef(num_diff=g.zeros(5, 3), DENS=c.state["DENS"], MOMZ=c.state["MOMZ"],
                                     MOMX=c.state["MOMX"], MOMY=c.state["MOMY"], RHOT=c.state["RHOT"], CDZ=g.CDZ,
                                     CDX=g.CDX, CDY=g.CDY, FDZ=g.FDZ, FDX=g.FDX, FDY=g.FDY, DT=0.5,
                                     REF_dens=c.ref["REF_dens"], REF_pott=c.ref["REF_pott"], ND_COEF=1e-3,
                                     ND_ORDER=2, ND_SFC_FACT=0.7, ND_USE_RS=True)
    assert e.value.code == 5
