"""The C-ABI library: every function declared in include/awcm_b200.h is exported, the Python
binding covers them, and without a GPU the library fails loudly (no CPU fallback)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "awcm_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**((?:awcm|euler)\w*)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("awcm2d_create", "awcm2d_step", "awcm2d_prepare", "awcm2d_manager", "awcm1d_batch_create",
              "awcm1d_batch_steps", "awcm1d_step_noalloc", "euler2d_flux", "awcm_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(awcm_lib):
    lib = awcm_lib.LIB_PATH
    assert os.path.exists(lib)
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing


def test_python_binding_covers_header(awcm_lib):
    bound = set(awcm_lib.exported_symbols())
    missing = [n for n in declared() if n not in bound]
    assert not missing, missing


def test_loads_and_reports_version(awcm_lib):
    assert b"sm_100a" in awcm_lib.load().awcm_version()


def test_fails_loudly_without_device(awcm_lib):
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(awcm_lib.AwcmError):
        awcm_lib.AWCM2D(4, 9, 9, 0.0, 1.0, 0.0, 1.0)


@pytest.mark.parametrize("name,args", [
    ("awcm1d_batch_run", (None, 1)),
    ("awcm1d_batch_steps", (None, 1)),
    ("awcm1d_batch_sync", (None,)),
    ("awcm1d_batch_set_launch", (None, 256, 0)),
])
def test_null_handle_is_an_argument_error(name, args, awcm_lib):
    """The batch entry points reject a null handle with AWCM_ERR_ARG before touching the device."""
    lib = awcm_lib.load()
    assert getattr(lib, name)(*args) == 1
