"""The C-ABI library without a GPU: it loads, exports every entry point the
header declares, answers the no-compute calls, and refuses (rather than
falling back to the CPU) when there is no device."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

from feicar_b200 import fg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "feicar_b200.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    L = fg.lib()
    names = _declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_status_strings():
    L = fg.lib()
    assert L.fg_version().decode().startswith("feicar-b200")
    for s in range(11):
        assert len(L.fg_status_string(s).decode()) > 0


def test_default_config_matches_reference_defaults():
    cfg = fg.default_config()
    assert cfg.precision == fg.FG_PREC_FP64
    assert (cfg.nu1, cfg.nu2) == (2, 2)
    assert cfg.rtol == 1e-8
    assert list(cfg.pbc) == [fg.FG_PBC_NEUMANN] * 6
    assert cfg.probe_length == 2.0 and cfg.probe_length_dead == 2.0
    assert cfg.gauge_corner == 1
    assert cfg.outer == fg.FG_OUTER_FGMRES and cfg.restart == 8


def test_null_and_bad_arguments_are_rejected():
    L = fg.lib()
    h = C.c_void_p()
    xs = np.linspace(0, 1, 9)
    p = xs.ctypes.data_as(C.c_void_p)
    # bad sizes / non-monotone nodes are refused before any device call
    assert L.fg_case_create(2, 9, 9, p, p, p, None, 0, C.byref(h)) == 5
    bad = xs[::-1].copy()
    pb = bad.ctypes.data_as(C.c_void_p)
    assert L.fg_case_create(9, 9, 9, pb, p, p, None, 0, C.byref(h)) == 5
    assert L.fg_solve_poisson(None, None, None, None, None, None, None) == 5
    assert L.fg_case_destroy(None) == 0


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    n = C.c_int(-1)
    fg.lib().fg_device_count(C.byref(n))
    assert n.value == 0
    from feicar_b200 import synth
    with pytest.raises(fg.FGError) as e:
        fg.Case(synth.small_grid(8, 8, 8))
    assert e.value.status == 8  # FG_NO_DEVICE


def test_momentum_and_boundary_entry_points_reject_missing_arguments():
    """The momentum iteration and outer-boundary entry points refuse a
    missing handle, array or parameter block before any device call."""
    L = C.CDLL(fg.lib()._name)  # its own function objects: the bindings' argtypes stay untouched
    vp = C.c_void_p
    f = L.fg_body_intercept_values_device
    f.restype = C.c_int
    f.argtypes = [vp, C.c_int, C.c_double] + [vp] * 4
    assert f(None, 1, 0.1, None, None, None, None) == 5
    for n, k in (("fg_itsolv_ad_device", 7), ("fg_calc_residual_ad_device", 9),
                 ("fg_set_outer_velocity_bc_device", 6), ("fg_set_outer_ghost_velocity_device", 5),
                 ("fg_enforce_global_mass_consv_device", 8),
                 ("fg_face_vel_device", 10), ("fg_update_pressure_device", 3)):
        f = getattr(L, n)
        f.restype = C.c_int
        f.argtypes = [vp] * k
        assert f(*([None] * k)) == 5, n  # FG_BAD_INPUT
    f = L.fg_solve_ad_device
    f.restype = C.c_int
    f.argtypes = [vp] * 15 + [C.c_int, C.c_double, C.c_int, C.c_double, vp]
    assert f(*([None] * 15), 10, 1e-10, 10, 1e-8, None) == 5
    f = L.fg_ghostcell_velocity_device
    f.restype = C.c_int
    f.argtypes = [vp] * 6 + [C.c_int, C.c_double, vp]
    assert f(*([None] * 6), 10, 1e-10, None) == 5
