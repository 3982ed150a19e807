"""The C-ABI library without a GPU: it loads, exports what the header declares,
and its host-side argument checks answer before any device work."""
import ctypes
import re

import pytest

from scale_b200 import hevi
from scale_b200.build import LIB, ROOT


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(LIB))
    declared = hevi.header_functions()
    assert len(declared) >= 18
    for name in declared:
        assert hasattr(lib, name), name


def test_header_declarations_cite_the_reference():
    text = (ROOT / "include" / "scale_hevi.h").read_text()
    for m in re.finditer(r"Replaces\s+(\w+)", text):
        assert m.group(1) in ("the",) or m.group(1).startswith(("ATMOS_DYN", "COMM_vars8")), m.group(1)
    assert "scale_atmos_dyn_tstep_short_fvm_hevi.F90:128-1089" in text


def _index(**over):
    d = dict(KA=24, IA=20, JA=16, KS=3, KE=22, IS=3, IE=18, JS=3, JE=14, KMAX=20, IMAX=16, JMAX=12,
             KHALO=2, IHALO=2, JHALO=2, IBLOCK=16, JBLOCK=12)
    d.update(over)
    return d


def test_setup_rejects_inconsistent_index_set():
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(KA=25))
    assert e.value.code == 1 and "inconsistent" in str(e.value)


def test_setup_rejects_unsupported_options():
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(), flux_type="UD7")
    assert e.value.code == 5
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(KA=24, IA=24, JA=20, IS=5, IE=20, JS=5, JE=16, IHALO=4, JHALO=4))
    assert e.value.code == 5 and "halo" in str(e.value)
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(IBLOCK=8))
    assert e.value.code == 5
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(KA=7, KMAX=3, KE=5))
    assert e.value.code == 5


def test_calls_before_setup_fail_cleanly():
    hevi.finalize()
    with pytest.raises(hevi.HeviError) as e:
        hevi.check()
    assert e.value.code == 2
    with pytest.raises(hevi.HeviError) as e:
        hevi.COMM_vars8_dev(None, 1)
    assert e.value.code == 2


def test_setup_without_device_reports_cuda_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index())
    assert e.value.code == 3


def test_fortran_blank_padded_scheme_names_are_accepted():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    # the name is parsed before the device query: padded names get past parsing
    with pytest.raises(hevi.HeviError) as e:
        hevi.setup(_index(), flux_type="CD4     ", flux_tracer_type="UD3 ")
    assert e.value.code == 3


def test_unknown_flux_scheme_rejected_before_device_work():
    """Scheme names outside UD3, CD4, UD3KOREN1993, CD2, UD5 and CD6 are
    refused before any device work."""
    from scale_b200 import hevi, mkinit

    g = mkinit.uniform_grid(8, 8, 8, 500.0, 500.0, 250.0)
    for name in ("UD1", "UD7", "CD8"):
        with pytest.raises(hevi.HeviError, match="not supported"):
            hevi.setup(g.index_dict(), name, "UD3")


def test_six_point_schemes_need_a_halo_of_three():
    """UD5 and CD6 read three points on each side: with IHALO = JHALO = 2 the
    setup fails before any device work (scale_atmos_dyn_fvm_flux.F90:742-749),
    for the dynamics and for the tracer scheme alike."""
    from scale_b200 import hevi, mkinit

    g2 = mkinit.uniform_grid(8, 8, 8, 500.0, 500.0, 250.0)
    for dyn, trc in (("UD5", "UD3"), ("CD6", "UD3"), ("UD3", "UD5")):
        with pytest.raises(hevi.HeviError, match="IHALO = JHALO = 3"):
            hevi.setup(g2.index_dict(), dyn, trc)
    g3 = mkinit.uniform_grid(8, 8, 8, 500.0, 500.0, 250.0, halo=3)
    assert (g3.IA, g3.IS, g3.IE) == (14, 4, 11)
    ens = [g3.index_dict(), g2.index_dict()]
    with pytest.raises(hevi.HeviError, match="one halo width"):
        hevi.ensemble_setup(ens, "UD3", "UD3")
