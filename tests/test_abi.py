"""The C-ABI library loads and exports every symbol include/*.h declares (CPU:
no compute calls)."""
import ctypes
import glob
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"HWYBLAS_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_the_reference_entry_points():
    names = declared_symbols()
    for s in ["dgemm_", "sgemm_", "dtrsm_", "dsyrk_", "idamax_", "dgetrf_", "dgetrf2_",
              "dlaswp_", "dgetrs_", "dgesv_", "dpotrf_", "dpotrf2_", "dpotrs_", "dposv_",
              "cblas_dgemm", "cblas_sgemm", "cblas_dtrsm", "cblas_idamax", "xerbla_",
              "hwyblas_set_error_handler"]:
        assert s in names, s


def test_library_exports_every_declared_symbol():
    import hwyblas_b200
    from hwyblas_b200 import _abi
    lib = hwyblas_b200.lib()
    names = declared_symbols()
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", hwyblas_b200.LIB_PATH],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = names - exported
    assert not missing, missing
    assert set(_abi.EXPORTED) == names


def test_library_has_no_oracle_dependency():
    """The product never links the oracle."""
    import hwyblas_b200
    out = subprocess.run(["ldd", hwyblas_b200.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out and "hwyref" not in out
    syms = subprocess.run(["nm", "-D", hwyblas_b200.LIB_PATH], capture_output=True,
                          text=True).stdout
    assert "orc_" not in syms
