"""The HEVI stage entry that allocates no device memory
(ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc), for callers that cannot let a
library allocate GPU memory, against the device entry of the library on the
same inputs over two consecutive calls. The file sorts last so that it also
runs after every other test in one session; it passes on its own in a fresh
process as well."""
import numpy as np
import pytest

import helpers
from scale_b200 import hevi

pytestmark = pytest.mark.gpu

NAMES = ("DENS_RK", "MOMZ_RK", "MOMX_RK", "MOMY_RK", "RHOT_RK", "mflx_hi", "tflx_hi")
# The entry remembers metric arrays it found flat by their device addresses. Every
# array this module hands it stays allocated until the module ends, so no later
# array (the non-flat metrics of the terrain test) can reuse a remembered address.
_KEEP = []


def _args(a, o):
    kw = dict(a)
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    return kw


def _dev(x):
    import torch

    if isinstance(x, np.ndarray) and x.ndim >= 2:
        t = torch.from_numpy(np.ravel(x, order="K").copy()).cuda()
        _KEEP.append(t)
        return t
    return x


def _outputs(g):
    import torch

    return {n: torch.zeros((3 if n.endswith("flx_hi") else 1) * g.KA * g.IA * g.JA, dtype=torch.float64,
                           device="cuda") for n in NAMES}


def _case(scheme):
    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20, stretched=True)
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    return g, c


@pytest.mark.parametrize("scheme", ["CD4", "UD3", "UD3KOREN1993"])
def test_no_alloc_stage_matches_device_entry(gpu, scheme):
    import torch

    g, c = _case(scheme)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        # a different state each call, so that a stale scratch would show
        ad = {k: _dev(v) for k, v in helpers.short_inputs(c, dtrk=0.5 + 0.25 * call, full=True).items()}
        o_na = _outputs(g)
        hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), scheme, stream, **_args(ad, o_na))
        torch.cuda.synchronize()

        hevi.setup(g.index_dict(), scheme, scheme)
        try:
            o_dev = _outputs(g)
            hevi.ATMOS_DYN_Tstep_short_fvm_hevi_dev(**_args(ad, o_dev))
            hevi.check()
        finally:
            hevi.finalize()
        for n in NAMES:
            got, want = o_na[n].cpu().numpy(), o_dev[n].cpu().numpy()
            # the same arithmetic on both sides: identical values
            assert helpers.same(got, want), f"call {call}: {n} differs (max abs {np.nanmax(np.abs(got - want)):.3e})"
        helpers.perturb_state(c, seed=8 + call)


def test_no_alloc_refuses_terrain_then_runs_flat(gpu):
    import torch

    g, c = _case("CD4")
    stream = torch.cuda.current_stream().cuda_stream
    a = helpers.short_inputs(c, full=False)
    hilly = {k: _dev(v) for k, v in a.items()}
    gs = a["GSQRT"].copy(order="F")
    gs[g.KS + 1, g.IS + 2, g.JS + 3, 0] = 1.01
    hilly["GSQRT"] = _dev(gs)
    with pytest.raises(hevi.HeviError) as e:
        hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), "CD4", stream, **_args(hilly, _outputs(g)))
    assert e.value.code == 5 and "terrain" in str(e.value)
    # the counter of non-flat values starts from zero again on the next call
    flat = {k: _dev(v) for k, v in a.items()}
    o = _outputs(g)
    hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), "CD4", stream, **_args(flat, o))
    torch.cuda.synchronize()
    assert all(torch.isfinite(o[n]).all() for n in NAMES)


def test_no_alloc_status_starts_clean_on_each_call(gpu):
    import torch

    g, c = _case("UD3")
    stream = torch.cuda.current_stream().cuda_stream
    a = helpers.short_inputs(c, full=True)
    bad = {k: _dev(v) for k, v in a.items()}
    rt = np.asfortranarray(a["RHOT_t"].copy())
    rt[g.KS + 2, g.IS + 1, g.JS + 1] = np.nan
    bad["RHOT_t"] = _dev(rt)
    with pytest.raises(hevi.HeviError) as e:
        hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), "UD3", stream, **_args(bad, _outputs(g)))
    assert e.value.code == 4
    good = {k: _dev(v) for k, v in a.items()}
    hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), "UD3", stream, **_args(good, _outputs(g)))


def test_no_alloc_rejects_a_domain_beyond_its_scratch(gpu):
    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20)
    idx = g.index_dict()
    # three (KA,IA,JA) fields above 32 MiB: the size check answers before any argument is read
    n = 512
    idx.update(IMAX=n, JMAX=n, IA=n + 4, JA=n + 4, IE=n + 2, JE=n + 2, IBLOCK=n, JBLOCK=n)
    with pytest.raises(hevi.HeviError) as e:
        hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(idx, "CD4", 0, divdmp_coef=0.0, CDZ=g.CDZ, FDZ=g.FDZ, FDX=g.FDX,
                                                     FDY=g.FDY, RCDZ=g.RCDZ, RCDX=g.RCDX, RCDY=g.RCDY, RFDZ=g.RFDZ,
                                                     RFDX=g.RFDX, RFDY=g.RFDY)
    assert e.value.code == 1 and "at most" in str(e.value)
