"""The C-ABI libraries load on a CPU-only machine and export every function
that include/tioga_b200.h declares (no compute calls: there is no GPU)."""
import ctypes as C
import os
import re

import pytest

from tests.conftest import ROOT, REF_LIB

HEADER = os.path.join(ROOT, "include", "tioga_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b((?:tioga|tioga_b200)_\w+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_tioga_api():
    names = declared_functions()
    for n in ["tioga_init_", "tioga_registergrid_data_", "tioga_registergrid_data_mb_",
              "tioga_preprocess_grids_", "tioga_performconnectivity_", "tioga_registersolution_",
              "tioga_dataupdate_mb_", "tioga_dataupdate_", "tioga_getdonorcount_",
              "tioga_getdonorinfo_", "tioga_delete_"]:
        assert n in names


def test_gpu_library_exports_every_declared_symbol():
    import tioga_b200
    lib = C.CDLL(tioga_b200.library_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_gpu_library_reports_missing_device_without_crashing():
    """On a machine without a GPU the library must refuse loudly (no CPU
    fallback) and keep the process alive."""
    import tioga_b200
    lib = tioga_b200.extras(C.CDLL(tioga_b200.library_path()))
    ok = lib.tioga_b200_device_ok()
    if ok:
        pytest.skip("a CUDA device is present")
    lib.tioga_init_(C.c_long(0))
    assert lib.tioga_b200_last_error() != 0


def test_reference_symbols_are_a_subset():
    """Every TIOGA entry point of the compiled reference that the header
    names is exported by the GPU library too (drop-in linking)."""
    if not os.path.exists(REF_LIB):
        pytest.skip("compiled reference not built here")
    import tioga_b200
    ref = C.CDLL(REF_LIB)
    gpu = C.CDLL(tioga_b200.library_path())
    for n in declared_functions():
        if n.startswith("tioga_b200"):
            continue
        assert hasattr(ref, n), f"{n} is not a reference symbol"
        assert hasattr(gpu, n)


def test_every_reference_entry_point_is_exported():
    """Drop-in linking: every tioga_* function of the compiled reference's C
    API is exported by the GPU library (the ones outside the accelerated path
    as "not supported" stubs)."""
    if not os.path.exists(REF_LIB):
        pytest.skip("compiled reference not built here")
    import subprocess
    import tioga_b200

    def exported(path):
        out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                             check=True).stdout
        return {ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-1].startswith("tioga_")}

    missing = sorted(exported(REF_LIB) - exported(tioga_b200.library_path()))
    assert not missing, missing


def test_unsupported_entry_points_report_without_a_gpu():
    """The AMR and p4est entry points return with an error status."""
    import tioga_b200
    lib = tioga_b200.extras(C.CDLL(tioga_b200.library_path()))
    lib.tioga_set_p4est_()
    assert lib.tioga_b200_last_error() != 0
    n = C.c_int(3)
    lib.tioga_register_amr_patch_count_(C.byref(n))
    assert lib.tioga_b200_last_error() != 0
