"""The HEVI stage entry that allocates no device memory
(ATMOS_DYN_Tstep_short_fvm_hevi_b200_noalloc) against the device entry of the
library, on the same inputs, over two consecutive calls. The file sorts last
so that it also runs after every other test in one session; it passes on its
own in a fresh process as well."""
import numpy as np
import pytest

import helpers
from scale_b200 import hevi

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same kernels on both sides: any difference beyond round-off is a bug


def _close(got, want):
    same_nan = np.array_equal(np.isnan(got), np.isnan(want))
    g, w = np.nan_to_num(got), np.nan_to_num(want)
    return same_nan and np.all(np.abs(g - w) <= RTOL * np.maximum(np.abs(w), 1e-300))


def _args(a, o):
    kw = dict(a)
    kw.update(o)
    kw.update(PROG_RK=None, PROG0=None, PROG=None, FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False,
              FLAG_FCT_ALONG_STREAM=True, BND_W=False, BND_E=False, BND_S=False, BND_N=False, last=False)
    return kw


def test_no_alloc_stage_matches_device_entry(gpu):
    import torch

    g = helpers.small_grid(IMAX=16, JMAX=12, KMAX=20, stretched=True)
    c = helpers.small_case(g, "CD4")
    helpers.perturb_state(c)

    def dev(x):
        return torch.from_numpy(np.ravel(x, order="K").copy()).cuda() if isinstance(x, np.ndarray) and x.ndim >= 2 else x

    names = ("DENS_RK", "MOMZ_RK", "MOMX_RK", "MOMY_RK", "RHOT_RK", "mflx_hi", "tflx_hi")
    sizes = {n: (3 if n.endswith("flx_hi") else 1) * g.KA * g.IA * g.JA for n in names}
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        # a different state each call, so that a stale scratch would show
        a = helpers.short_inputs(c, dtrk=0.5 + 0.25 * call, full=True)
        ad = {k: dev(v) for k, v in a.items()}
        o_na = {n: torch.zeros(sizes[n], dtype=torch.float64, device="cuda") for n in names}
        hevi.ATMOS_DYN_Tstep_short_fvm_hevi_noalloc(g.index_dict(), "CD4", stream, **_args(ad, o_na))
        torch.cuda.synchronize()

        hevi.setup(g.index_dict(), "CD4", "CD4")
        try:
            o_dev = {n: torch.zeros(sizes[n], dtype=torch.float64, device="cuda") for n in names}
            hevi.ATMOS_DYN_Tstep_short_fvm_hevi_dev(**_args(ad, o_dev))
            hevi.check()
        finally:
            hevi.finalize()
        for n in names:
            got, want = o_na[n].cpu().numpy(), o_dev[n].cpu().numpy()
            assert _close(got, want), f"call {call}: {n} differs (max abs {np.nanmax(np.abs(got - want)):.3e})"
        helpers.perturb_state(c)


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
