"""The C ABI library loads without a GPU and exports every symbol include/impact_b200.h declares."""
import os
import re

import impact_b200 as I

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "impact_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)
    skip = {"if", "for", "while", "return", "sizeof", "defined"}
    return sorted({n for n in names if n not in skip and (n.endswith("_") or n.startswith("impact_b200_"))})


def test_header_declares_reference_launchers():
    syms = declared_symbols()
    for ref in ["gradient_launcher_", "divergence_launcher_", "divergence2_launcher_", "helmholtz_explicit_launcher_",
                "nonlinear_upwind_launcher_", "interpolate2_pre_vel_launcher_", "interpolate2_vel_pre_launcher_",
                "axpby_launcher_", "jor_launcher_", "get_ghost_launcher_", "pressure_bc_launcher_",
                "jacobi_launcher_", "product_dg_relax_launcher_"]:
        assert ref in syms


def test_library_exports_every_declared_symbol():
    L = I.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_host_side_calls_without_gpu():
    assert I.lib().impact_b200_version() >= 10000
    g = I.Grid((17, 17, 17))
    assert g.tab["cdg"][0].shape == (3 * 17,)
    assert I.Case.bytes_needed((17, 17, 17), 0) > I.Case.bytes_needed((17, 17, 17), 1) > 0


def test_case_entry_points_reject_a_null_case_without_touching_the_gpu():
    """The case entry points added for transfers, snapshots and the inflow waveform validate their
    arguments before any CUDA call: a null case is an error with a message, never a crash."""
    import ctypes as C

    L = I.lib()
    buf = (C.c_double * 4)()
    fields = (C.c_int * 1)(0)
    ptrs = (C.POINTER(C.c_double) * 1)(buf)
    calls = [
        ("impact_b200_case_upload_async", lambda: L.impact_b200_case_upload_async(None, 0, buf, 0, 1, None)),
        ("impact_b200_case_download_async", lambda: L.impact_b200_case_download_async(None, 0, buf, 0, 1, None)),
        ("impact_b200_case_defer_pressure", lambda: L.impact_b200_case_defer_pressure(None, None)),
        ("impact_b200_case_set_inflow_waveform",
         lambda: L.impact_b200_case_set_inflow_waveform(None, 2, buf, buf)),
        ("impact_b200_case_snapshot", lambda: L.impact_b200_case_snapshot(None, 1, fields, ptrs, None)),
        ("impact_b200_case_synchronize", lambda: L.impact_b200_case_synchronize(None)),
        ("impact_b200_case_set_markers", lambda: L.impact_b200_case_set_markers(None, 1, buf, None, 0.1, 2)),
        ("impact_b200_case_ibm_interpolate", lambda: L.impact_b200_case_ibm_interpolate(None, buf)),
        ("impact_b200_case_ibm_spread", lambda: L.impact_b200_case_ibm_spread(None, buf, buf, 8)),
    ]
    for name, call in calls:
        assert call() != 0, name
        assert name in I.last_error(), (name, I.last_error())


def test_pressure_bc_plane_switch_host_side():
    """The plane switch is host state only: it round-trips without a GPU and rejects other modes."""
    assert I.pressure_bc_plane() == 0
    I.set_pressure_bc_plane(1)
    try:
        assert I.pressure_bc_plane() == 1
    finally:
        I.set_pressure_bc_plane(0)
    import pytest

    with pytest.raises(I.ImpactError, match="mode 0"):
        I.set_pressure_bc_plane(2)
    I.lib().impact_b200_clear_error()
    assert I.pressure_bc_plane() == 0
