"""The C ABI: the library loads and exports every entry point include/mdb.h
declares, and the ctypes mirror matches the header.  No compute calls: these
run without a GPU."""

from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_functions() -> list[str]:
    text = (ROOT / "include" / "mdb.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*|void)\s+(mdb_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    import importlib.util
    import sys

    spec = importlib.util.spec_from_file_location("mdb_build", ROOT / "making-it-rain-webgpu_b200" / "build.py")
    build = importlib.util.module_from_spec(spec)
    sys.modules["mdb_build"] = build
    spec.loader.exec_module(build)
    build.build()
    from mdb200 import abi

    return abi.load()


def test_header_declares_the_boundary():
    names = header_functions()
    for want in ("mdb_create", "mdb_batch_create", "mdb_run", "mdb_evaluate", "mdb_potential",
                 "mdb_get_positions", "mdb_set_box", "mdb_destroy", "mdb_last_error"):
        assert want in names


def test_library_exports_every_declared_symbol(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_ctypes_mirror_covers_the_header():
    from mdb200 import abi

    assert set(abi.EXPORTS) == set(header_functions())


def test_abi_version_and_status_strings(lib):
    from mdb200 import abi

    assert lib.mdb_abi_version() == abi.ABI_VERSION
    assert lib.mdb_status_string(abi.ERR_CUTOFF_TOO_LARGE_FOR_BOX) == b"cutoff too large for box"
    assert lib.mdb_status_string(12345) == b"unknown status"


def test_struct_layouts_match_the_header():
    """Field offsets the C compiler would give, checked by ctypes arithmetic."""
    from mdb200 import abi

    assert C.sizeof(abi.Energies) == 8 * (18 + 9 + 1 + 9)
    assert abi.SystemDesc.box.offset == 16
    assert abi.StateDesc.box.offset == 16
    assert abi.RunOptions.seed.offset == 32


def test_null_arguments_are_refused_without_a_device(lib):
    from mdb200 import abi

    assert lib.mdb_create(None, None, None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_run(None, 1) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_destroy(None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.mdb_last_error(None) == b"no engine"
