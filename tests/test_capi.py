"""The C ABI library on the CPU: it loads, exports every symbol the header declares, and its
host-only set-up helpers agree with the reference's fixtures.  No GPU compute here."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden

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


def test_vector_files_match_the_reference_bytes(dh, orc, tmp_path):
    # RealVector::WriteVector / ReadVector: the reference's files read back exactly, and the same
    # components written by the library give the same bytes
    z = golden("disk_ground_n7_2s18_lz2.npz")
    for i, name in enumerate(z["interrupted_names"]):
        if not str(name).startswith("vector"):
            continue
        ref = bytes(z["interrupted_f%d" % i])
        p = tmp_path / str(name)
        p.write_bytes(ref)
        assert dh.vector_file_dimension(str(p)) == 1646
        x = dh.ReadVector(str(p))
        assert np.array_equal(x, orc.read_vector_bytes(ref))
        q = tmp_path / ("copy_" + str(name))
        dh.WriteVector(x, str(q))
        assert q.read_bytes() == ref
        assert not (tmp_path / ("copy_" + str(name) + ".tmp")).exists()


def test_vector_file_forms_and_errors(dh, tmp_path):
    x = np.random.default_rng(3).standard_normal(37)
    # the int64 form (int32 -1, then the dimension) that the reference writes from 2^31 on
    p = tmp_path / "large_form.vec"
    p.write_bytes(np.int32(-1).tobytes() + np.int64(37).tobytes() + x.tobytes())
    assert dh.vector_file_dimension(str(p)) == 37
    assert np.array_equal(dh.ReadVector(str(p)), x)
    # empty vector
    e = tmp_path / "empty.vec"
    dh.WriteVector(np.zeros(0), str(e))
    assert e.read_bytes() == np.int32(0).tobytes() and dh.ReadVector(str(e)).size == 0
    # missing, truncated, too long, wrong dimension for the buffer
    with pytest.raises(dh.DiagHamError, match="error -7"):
        dh.ReadVector(str(tmp_path / "missing.vec"))
    t = tmp_path / "truncated.vec"
    t.write_bytes(np.int32(37).tobytes() + x[:30].tobytes())
    with pytest.raises(dh.DiagHamError, match="do not hold"):
        dh.ReadVector(str(t))
    t.write_bytes(np.int32(37).tobytes() + np.concatenate([x, x[:1]]).tobytes())
    with pytest.raises(dh.DiagHamError, match="do not hold"):
        dh.ReadVector(str(t))
    with pytest.raises(dh.DiagHamError, match="expected 36"):
        dh.ReadVector(str(p), out=np.zeros(36))
    with pytest.raises(dh.DiagHamError, match="error -7"):
        dh.WriteVector(x, str(tmp_path / "no_such_dir" / "x.vec"))


def test_eigenstate_file_name(dh):
    # FQHE/docs/DataFormat/FermionOnSphere.xml:9-16; QHEOnSphereMainTask.cc:891
    assert dh.eigenstate_file_name("fermions", "coulomb", 8, 21, 0, 0) == "fermions_coulomb_n_8_2s_21_lz_0.0.vec"


def test_complex_vector_files_match_the_reference(dh, tmp_path):
    # a file written by the reference's ComplexVector::WriteVector (its product in the L = 8, K = 1
    # momentum sector): read back exactly, and written again byte for byte
    ref_file = os.path.join(GOLDEN, "complexvector_translations_L8_sz0_k1.vec")
    y = golden("translations_complex_L8_sz0_k1_j2_0.5.npz")["y"]
    z = dh.ReadComplexVector(ref_file)
    assert z.dtype == np.complex128 and np.array_equal(z, y)
    out = str(tmp_path / "again.vec")
    dh.WriteVector(z, out)
    assert open(out, "rb").read() == open(ref_file, "rb").read()
    # a complex file is not a real vector of the same length, nor the other way round
    with pytest.raises(dh.DiagHamError, match="error -7"):
        dh.ReadVector(ref_file)
    real = str(tmp_path / "real.vec")
    dh.WriteVector(np.arange(5.0), real)
    with pytest.raises(dh.DiagHamError, match="error -7"):
        dh.ReadComplexVector(real)


def test_spectrum_file_in_the_reference_layout(dh, tmp_path):
    # QHEOnSphereMainTask's spectrum file: header, "LValue/2 E" lines at 14 significant digits, LValue/2
    # truncated toward zero, the energy shift removed, optional <H> and <L^2> <L> columns; an existing
    # file is backed up as .bak, then .bak1
    name = str(tmp_path / dh.spectrum_file_name("fermions", "coulomb", 8, 21))
    assert name.endswith("fermions_coulomb_n_8_2s_21_lz.dat")
    f = dh.QHEOnSphereSpectrumFile(name)
    f.add(0, [13.914890702090714, -0.5])
    f.add(-3, [1.25e-20], energy_shift=-1.0)
    assert open(name).read() == "# Lz E\n0 13.914890702091\n0 -0.5\n-1 1\n"
    g = dh.QHEOnSphereSpectrumFile(name, energy_column=True, l_value_columns=True)
    g.add(4, [2.0], expectations=[2.0 + 1e-15], l2_values=[6.0])
    assert open(name).read() == "# Lz E <H> <L^2> <L>\n2 2 2 6 2\n"
    assert open(name + ".bak").read().startswith("# Lz E\n0 13.914890702091")
    dh.QHEOnSphereSpectrumFile(name)
    assert open(name + ".bak1").read().startswith("# Lz E <H>")


@pytest.mark.parametrize("make, pattern", [
    (lambda dh: dh.FermionOnSphere(0, 0, 8), "nbr_fermions must be >= 1"),
    (lambda dh: dh.FermionOnSphere(10, 0, 8), "do not fit in 9 orbitals"),
    (lambda dh: dh.FermionOnSphere(4, 0, 63), "FermionOnSphereLong takes up to 126"),
    (lambda dh: dh.FermionOnSphereLong(4, 0, 127), r"not in 1\.\.126"),
    (lambda dh: dh.FermionOnSphereLong(3, 1, 64), "not reachable"),
    (lambda dh: dh.BosonOnSphereShort(0, 0, 4), "nbr_bosons must be >= 1"),
    (lambda dh: dh.BosonOnSphereShort(10, 0, 54), "needs the reference's BosonOnSphere"),
    (lambda dh: dh.BosonOnSphereShort(3, 1, 4), "not reachable"),
    (lambda dh: dh.BosonOnSphereShort(2, 10, 4), "not reachable"),
    (lambda dh: dh.Spin1_2Chain(8, 1), "not reachable with 8 spins"),
    (lambda dh: dh.Spin1_2ChainWithTranslations(2, 0, 0), r"not in 3\.\.32"),
    (lambda dh: dh.Spin1_2ChainWithTranslations(33, 0, 1), r"not in 3\.\.32"),
    (lambda dh: dh.Spin1_2ChainWithTranslations(8, 8, 0), r"momentum 8 not in 0\.\.7"),
    (lambda dh: dh.Spin1_2ChainWithTranslations(8, 0, 3), "not reachable with 8 spins"),
])
def test_constructor_limits_are_codes(dh, make, pattern):
    """Every space constructor checks its sector before touching the device: the error is a status
    code with a message, on a machine without a GPU as on one with it."""
    with pytest.raises(dh.DiagHamError, match=pattern):
        make(dh)


def test_null_handles_are_codes(dh):
    lib = dh.load()
    d = ctypes.c_int64(-1)
    assert lib.dh_space_get_dimension(None, ctypes.byref(d)) != 0
    assert "null" in lib.dh_last_error().decode()
    assert lib.dh_fermion_on_sphere_create(4, 0, 8, 0, None) != 0
    assert "null output handle" in lib.dh_last_error().decode()


def test_missing_library_fails_loudly():
    """Without the built CUDA library the package raises on first use: there is no host fallback."""
    import subprocess
    import sys
    code = ("import diagham_b200 as dh\n"
            "dh._LIB_PATH = '/nonexistent/libdiagham_b200.so'\n"
            "try:\n"
            "    dh.FermionOnSphere(4, 0, 8)\n"
            "except dh.DiagHamError as e:\n"
            "    print('raised:', e)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "raised: libdiagham_b200.so is not built" in out.stdout


def test_every_entry_cites_its_reference_interface():
    """Each declared entry's comment gives the reference interface it replaces as file:line, or says
    that it has no reference counterpart; only the library's own utilities are exempt."""
    text = open(HEADER).read()
    utilities = {"dh_last_error", "dh_version", "dh_device_count", "dh_space_destroy", "dh_hamiltonian_destroy",
                 "dh_lanczos_destroy"}
    uncited = []
    for m in re.finditer(r"\b(dh_[a-z0-9_]+)\s*\(", text):
        before = text[:m.start()]
        if before.count("/*") > before.count("*/") or m.group(1) in utilities:
            continue
        comment = before[before.rfind("/*"):before.rfind("*/")]
        if not re.search(r"\.(cc|h):\d+|[Nn]o[\s*]+(reference[\s*]+)?counterpart", comment):
            uncited.append(m.group(1))
    assert not uncited, uncited
