"""FP64 budget sums on the device: the mass total (check_mass,
scale_atmos_dyn.F90:530-688) and the dry-air energy totals ENGT, ENGP, ENGK,
ENGI (mod_atmos_vars.F90:2097-2171) against the oracle on the same state."""
import numpy as np
import pytest

import helpers
import oracle
from scale_b200 import hevi

pytestmark = pytest.mark.gpu

# the totals sum the same cell values in another order (column sums, then a
# tree over columns); the temperature goes through pow(), whose last bit may
# differ between glibc and CUDA
RTOL = 1e-12


def _dev(x):
    import torch

    return torch.from_numpy(np.ravel(x, order="K").copy()).cuda()


@pytest.mark.parametrize("scheme", ["UD3", "CD4"])
def test_energy_and_mass_totals_match_the_oracle(gpu, scheme):
    g = helpers.small_grid(IMAX=20, JMAX=14, KMAX=24, stretched=True)
    c = helpers.small_case(g, scheme)
    helpers.perturb_state(c)
    want = oracle.energy_sum(g, c.state, g.CZ)
    m_want = oracle.domain_sum(g, c.state["DENS"])
    hevi.setup(g.index_dict(), scheme, scheme)
    try:
        d = {n: _dev(c.state[n]) for n in ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")}
        got = hevi.energy_sum_dev(**d, CZ=g.CZ, CDZ=g.CDZ, CDX=g.CDX, CDY=g.CDY)
        m_got = hevi.domain_sum_dev(d["DENS"], g.CDZ, g.CDX, g.CDY)
    finally:
        hevi.finalize()
    for n in want:
        assert abs(got[n] - want[n]) <= RTOL * abs(want["ENGT"]), (n, got[n], want[n])
    assert abs(m_got - m_want) <= RTOL * m_want
