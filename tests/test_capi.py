"""The C ABI library on the CPU: it loads, exports every symbol the header declares, and its
host-only set-up helpers agree with the reference's fixtures.  No GPU compute here."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden

HEADER = os.path.join(ROOT, "include", "diagham_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dh_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "dh_hamiltonian_low_level_add_multiply" in names and "dh_lanczos_run" in names
    assert len(names) >= 35


def test_library_exports_every_declared_symbol(dh):
    lib = ctypes.CDLL(dh.library_path())
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers exactly the declared set
    assert sorted(dh.SIGNATURES) == declared_symbols()


def test_version_and_device_count(dh):
    assert "sm_100a" in dh.version()
    assert dh.device_count() >= 0


@pytest.mark.parametrize("two_s", [8, 21, 27, 33])
def test_coulomb_pseudopotentials_host(dh, two_s):
    ref = golden("pseudopotentials_2s%d.npz" % two_s)["v"]
    v = dh.coulomb_pseudopotentials(two_s)
    assert np.max(np.abs(v - ref) / np.abs(ref)) < 1e-13


def test_clebsch_gordan_host(dh, orc):
    for args in [(33, 1, 33, -1, 0), (33, 5, 33, 3, 20), (21, -7, 21, 9, 14), (8, 2, 4, -2, 6)]:
        assert abs(dh.clebsch_gordan(*args) - orc.clebsch_gordan(*args)) < 1e-14


def test_errors_are_codes_not_aborts(dh):
    # invalid sector parity is rejected before any device work
    with pytest.raises(dh.DiagHamError, match="not reachable"):
        dh.FermionOnSphere(5, 1, 12)
    with pytest.raises(dh.DiagHamError):
        dh.Spin1_2Chain(40, 0)
    msg = dh.load().dh_last_error().decode()
    assert "chain length" in msg
