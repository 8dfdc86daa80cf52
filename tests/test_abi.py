"""The C-ABI library: it loads without a GPU, exports every entry point that
include/msb200.h declares, and its struct layouts agree with the Python
binding.  No compute call runs here."""

import ctypes
import re
import subprocess
import textwrap

import pytest

from microsimulator_b200 import abi
from tests.conftest import ROOT

HEADER = ROOT / "include" / "msb200.h"


def declared_functions():
    text = HEADER.read_text()
    names = re.findall(r"^\s*(?:int|void|size_t|uint64_t|const char\*)\s+(msb_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    assert "msb_find_cell_contacts" in names
    assert "msb_solve_contact_forces" in names
    assert "msb_advance_contact_dynamics" in names
    assert set(names) <= set(abi.SIGNATURES) | set(names)


def test_library_exports_every_declared_symbol():
    library = abi.load_library()
    for name in declared_functions():
        assert hasattr(library, name), name
        assert name in abi.SIGNATURES, name


def test_device_count_needs_no_gpu():
    library = abi.load_library()
    assert int(library.msb_device_count()) >= 0


def test_struct_layouts_match_the_header(tmp_path):
    probe = tmp_path / "sizes.c"
    probe.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "{HEADER}"
        int main(void) {{
          printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",
            sizeof(msb_cell_contact), sizeof(msb_external_contact), sizeof(msb_contact_row),
            sizeof(msb_contact_body), sizeof(msb_constraint), sizeof(msb_contact_system),
            sizeof(msb_contact_dynamics_parameters), sizeof(msb_contact_dynamics_report),
            sizeof(msb_cell_arrays), offsetof(msb_contact_system, dt));
          return 0;
        }}
    """))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c11", str(probe), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    expected = [
        ctypes.sizeof(abi.CellContact),
        ctypes.sizeof(abi.ExternalContact),
        ctypes.sizeof(abi.ContactRow),
        ctypes.sizeof(abi.ContactBody),
        ctypes.sizeof(abi.Constraint),
        ctypes.sizeof(abi.ContactSystem),
        ctypes.sizeof(abi.ContactDynamicsParameters),
        ctypes.sizeof(abi.ContactDynamicsReport),
        ctypes.sizeof(abi.CellArrays),
        abi.ContactSystem.dt.offset,
    ]
    assert sizes == expected


def test_status_mapping_mirrors_reference_exceptions():
    with pytest.raises(ValueError):
        abi.raise_for_status(abi.ERR_INVALID_ARGUMENT, "bad")
    with pytest.raises(OverflowError):
        abi.raise_for_status(abi.ERR_OVERFLOW, "big")
    with pytest.raises(RuntimeError):
        abi.raise_for_status(abi.ERR_RUNTIME, "failed")
    abi.raise_for_status(abi.OK, "")


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(FileNotFoundError):
        abi.load_library(tmp_path / "libmsb200.so")
