"""Disk storage of the Lanczos state in the reference's formats (BasicLanczosAlgorithmWithDiskStorage,
BasicLanczosAlgorithmWithGroundStateDiskStorage) on N=7 2S=18 2Lz=2:

- the checkpoint after 14 iterations against the files the reference wrote after the same iterations
  from the same start vector (fields exact, tridiagonal and Lanczos vectors to 1e-12, H v to 1e-11);
- resuming from the reference's files ends where the reference's resumed run ends (energy 1e-12,
  iteration counter within 2), also from a state written in the middle of the reference's
  ground-state assembly.  Ground states are compared by overlap (1 - |<a|b>| < 1e-7) and Rayleigh
  quotient (1e-7 relative): a Ritz vector rebuilt by replaying the recurrence from the start vector
  moves by ~1e-9 in overlap under a 1e-15 change of that vector on this sector (gap 0.021), and the
  reference's own ground state is 1.1e-9 from the exact one in overlap;
- the reference resumes from our files (when its compiled harness is present) to its own result;
- an interrupted and resumed run here equals the uninterrupted one (FP64 and FP32 products);
- checkpoint interval, device vectors in vector files, and the error cases."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu

N, S, LZ = 7, 18, 2
TOOL = os.path.join(ROOT, "oracle", "_ref", "ref_tool")


def _fixture(fmt):
    return golden("disk_%s_n7_2s18_lz2.npz" % fmt)


def _files(z, prefix):
    return {str(n): bytes(z["%s_f%d" % (prefix, i)]) for i, n in enumerate(z["%s_names" % prefix])}


def _hamiltonian(gpu, z, precision="fp64"):
    sp = gpu.FermionOnSphere(N, LZ, S)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, N, S, z["v"])
    H.set_precision(precision)
    return H


def _lanczos(gpu, fmt, H, directory, interval=1, max_iter=400):
    if fmt == "basic":
        return gpu.BasicLanczosAlgorithmWithDiskStorage(H, 1, max_iter, directory=str(directory), interval=interval)
    return gpu.BasicLanczosAlgorithmWithGroundStateDiskStorage(H, max_iter, directory=str(directory),
                                                               interval=interval)


def _state(orc, d, fmt):
    return orc.read_lanczos_state((d / "lanczos.dat").read_bytes(), fmt)


def _vectors(orc, d, st, fmt):
    names = st["names"] if fmt == "basic" else ["vector.1", "vector.2", "vector.3"]
    return [orc.read_vector_bytes((d / n).read_bytes()) for n in names]


def _overlap_error(a, b):
    return abs(1.0 - abs(float(a @ b)) / (np.linalg.norm(a) * np.linalg.norm(b)))


def _check_ground_state(H, psi, psi_ref, e_ref):
    assert _overlap_error(psi, psi_ref) < 1e-7
    assert abs(H.MatrixElement(psi, psi) - e_ref) <= 1e-7 * abs(e_ref)


@pytest.mark.parametrize("fmt", ["basic", "ground"])
def test_checkpoint_matches_reference_files(gpu, orc, tmp_path, fmt):
    z = _fixture(fmt)
    H = _hamiltonian(gpu, z)
    lz = _lanczos(gpu, fmt, H, tmp_path)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), H.dim))
    r = lz.solve(max_iter=int(z["stop"]))  # the reference's loop stopped by --nbr-iter 14
    assert r["iterations"] == int(z["stop"]) and not r["converged"]
    ref_files = _files(z, "interrupted")
    ref = orc.read_lanczos_state(ref_files["lanczos.dat"], fmt)
    ours = _state(orc, tmp_path, fmt)
    for k in ("index", "nbr_row", "precision", "ground_flag"):
        assert ours[k] == ref[k], k
    assert abs(ours["prev_last"] - ref["prev_last"]) <= 1e-12 * abs(ref["prev_last"])
    scale = np.max(np.abs(ref["diag"]))
    assert np.max(np.abs(ours["diag"] - ref["diag"])) <= 1e-12 * scale
    assert np.max(np.abs(ours["upper"] - ref["upper"])) <= 1e-12 * scale
    names = ref["names"] if fmt == "basic" else ["vector.1", "vector.2", "vector.3"]
    for q, (mine, n) in enumerate(zip(_vectors(orc, tmp_path, ours, fmt), names)):
        theirs = orc.read_vector_bytes(ref_files[n])
        tol = 1e-12 if q < 2 else 1e-11  # the third vector is H v: rounding grows with |H|
        assert np.max(np.abs(mine - theirs)) <= tol * max(1.0, np.max(np.abs(theirs))), n
    if fmt == "ground":
        v0 = orc.read_vector_bytes((tmp_path / "vector.0").read_bytes())
        assert np.max(np.abs(v0 - orc.read_vector_bytes(ref_files["vector.0"]))) < 1e-15
    assert not [p for p in os.listdir(tmp_path) if p.endswith(".tmp")]


@pytest.mark.parametrize("fmt", ["basic", "ground"])
def test_resume_from_reference_files(gpu, orc, tmp_path, fmt):
    z = _fixture(fmt)
    for name, b in _files(z, "interrupted").items():
        (tmp_path / name).write_bytes(b)
    H = _hamiltonian(gpu, z)
    lz = _lanczos(gpu, fmt, H, tmp_path)
    lz.ResumeLanczosAlgorithm()
    assert not lz.TestConvergence()
    r = lz.solve(max_iter=400)
    e_ref = float(z["resumed_eigenvalue"])
    assert r["converged"] and abs(r["eigenvalues"][0] - e_ref) <= 1e-12 * abs(e_ref)
    assert abs(r["iterations"] - int(z["resumed_iterations"])) <= 2
    if fmt == "ground":
        _check_ground_state(H, lz.GetGroundState(), z["psi"], e_ref)
    else:
        # the basic format does not store the start vector
        with pytest.raises(gpu.DiagHamError, match="start vector"):
            lz.GetGroundState()


def test_ground_state_from_reference_assembly_state(gpu, orc, tmp_path):
    # the reference stopped while assembling its ground state (GroundStateEvaluationFlag 1): the
    # finished run's matrix and vector.0 rebuild the ground state here
    z = _fixture("ground")
    for name, b in _files(z, "assembly").items():
        (tmp_path / name).write_bytes(b)
    H = _hamiltonian(gpu, z)
    lz = _lanczos(gpu, "ground", H, tmp_path)
    lz.ResumeLanczosAlgorithm()
    assert lz.TestConvergence()
    e_ref = float(z["full_eigenvalue"])
    assert abs(lz.GetGroundStateEnergy() - e_ref) <= 1e-13 * abs(e_ref)
    _check_ground_state(H, lz.GetGroundState(), z["psi"], e_ref)
    with pytest.raises(gpu.DiagHamError, match="error -6"):
        lz.RunLanczosAlgorithm(1)


@pytest.mark.skipif(not os.path.exists(TOOL), reason="the reference harness is not built here")
@pytest.mark.parametrize("fmt", ["basic", "ground"])
def test_reference_resumes_from_our_files(gpu, orc, tmp_path, fmt):
    z = _fixture(fmt)
    H = _hamiltonian(gpu, z)
    d = tmp_path / "state"
    d.mkdir()
    lz = _lanczos(gpu, fmt, H, d)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), H.dim))
    lz.solve(max_iter=int(z["stop"]))
    vf = tmp_path / "v.bin"
    np.asarray(z["v"], np.float64).tofile(str(vf))
    out = tmp_path / "l.out"
    subprocess.run([TOOL, "fqhe_lanczos_disk", str(N), str(S), str(LZ), str(vf), fmt, "400", "0", str(d), "resume",
                    "100000", str(out), "-"], check=True, stdout=subprocess.DEVNULL, timeout=600)
    b = out.read_bytes()
    it = int(np.frombuffer(b[4:8], np.int32)[0])
    e = float(np.frombuffer(b[20:28], np.float64)[0])
    e_ref = float(z["full_eigenvalue"])
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
    assert abs(it - int(z["resumed_iterations"])) <= 2


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("fmt", ["basic", "ground"])
def test_interrupted_run_resumes_to_the_uninterrupted_result(gpu, orc, tmp_path, fmt, precision):
    z = _fixture(fmt)
    H = _hamiltonian(gpu, z, precision)
    x0 = orc.random_vector(5, H.dim)
    cls = gpu.BasicLanczosAlgorithm if fmt == "basic" else gpu.BasicLanczosAlgorithmWithGroundState
    a = cls(H, 1, 400)
    a.InitializeLanczosAlgorithm(x0)
    ra = a.solve(max_iter=400)
    psi_a = a.GetGroundState() if fmt == "ground" else None
    b = _lanczos(gpu, fmt, H, tmp_path, interval=4)
    b.InitializeLanczosAlgorithm(x0)
    rb = b.solve(max_iter=21)
    assert not rb["converged"]
    del b
    c = _lanczos(gpu, fmt, H, tmp_path)
    c.ResumeLanczosAlgorithm()
    rc = c.solve(max_iter=400)
    assert rc["converged"] and rb["iterations"] + rc["iterations"] == ra["iterations"]
    e = ra["eigenvalues"][0]
    assert abs(rc["eigenvalues"][0] - e) <= 1e-13 * abs(e)
    if fmt == "ground":
        assert _overlap_error(c.GetGroundState(), psi_a) < 1e-12


def test_checkpoint_interval_and_name_sets(gpu, orc, tmp_path):
    z = _fixture("basic")
    H = _hamiltonian(gpu, z)
    lz = _lanczos(gpu, "basic", H, tmp_path, interval=5)
    lz.InitializeLanczosAlgorithm(orc.random_vector(1, H.dim))
    lz.RunLanczosAlgorithm(3)
    assert not (tmp_path / "lanczos.dat").exists()  # 3 rows < interval
    lz.RunLanczosAlgorithm(1)
    lz.WriteState()
    st = _state(orc, tmp_path, "basic")
    assert st["index"] == 2 and st["nbr_row"] == 4
    r = lz.solve(max_iter=30)  # a continued run: the driver's first call adds 3 rows
    m, rows = lz.counters()
    st = _state(orc, tmp_path, "basic")
    assert st["index"] == rows - 2 and st["nbr_row"] == rows
    assert set(os.listdir(tmp_path)) <= {"lanczos.dat"} | {"vector%d" % k for k in range(1, 7)}
    v1, v2, v3 = _vectors(orc, tmp_path, st, "basic")
    assert abs(v2 @ v2 - 1.0) < 1e-13 and abs(st["diag"][-1] - v2 @ v3) < 1e-12 * abs(st["diag"][-1])
    assert r["iterations"] > 0


def test_device_vectors_in_vector_files(gpu, tmp_path):
    import torch
    x = torch.rand(1000, dtype=torch.float64, device="cuda")
    p = str(tmp_path / "x.vec")
    gpu.WriteVector(x, p)
    y = torch.zeros_like(x)
    gpu.ReadVector(p, out=y)
    assert torch.equal(x, y)
    assert np.array_equal(gpu.ReadVector(p), x.cpu().numpy())


def test_disk_storage_errors(gpu, orc, tmp_path):
    z = _fixture("basic")
    H = _hamiltonian(gpu, z)
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu.FullReorthogonalizedLanczosAlgorithm(H, 1, 100).set_disk_storage(str(tmp_path))
    lz = _lanczos(gpu, "basic", H, tmp_path)
    with pytest.raises(gpu.DiagHamError, match="error -7"):
        lz.ResumeLanczosAlgorithm()  # nothing on disk
    lz.InitializeLanczosAlgorithm(orc.random_vector(2, H.dim))
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        lz.solve_refined(max_iter=100, precision=1e-12)
    # a ground-state-format state is not a basic one
    g = _fixture("ground")
    d = tmp_path / "g"
    d.mkdir()
    for name, b in _files(g, "interrupted").items():
        (d / name).write_bytes(b)
    with pytest.raises(gpu.DiagHamError, match="error -7"):
        _lanczos(gpu, "basic", H, d).ResumeLanczosAlgorithm()
    # more stored rows than the handle holds
    with pytest.raises(gpu.DiagHamError, match="error -1"):
        _lanczos(gpu, "ground", H, d, max_iter=8).ResumeLanczosAlgorithm()
    # a directory that cannot be written: the error comes back from the call that waits for the files
    bad = _lanczos(gpu, "ground", H, tmp_path / "missing")
    with pytest.raises(gpu.DiagHamError, match="error -7"):
        bad.InitializeLanczosAlgorithm(orc.random_vector(2, H.dim))
        bad.RunLanczosAlgorithm(3)
        bad.WriteState()


@pytest.mark.parametrize("space", ["fermions_2s70", "bosons_2s45"])
def test_disk_storage_on_the_wider_spaces(gpu, orc, tmp_path, space):
    # checkpoint/resume is the same on the 128-bit fermion engine (FermionOnSphereLong N=4 2S=70) and on
    # bosons beyond 41-bit words (BosonOnSphereShort N=4 2S=45): an interrupted ground-state run resumed
    # from its files ends where the uninterrupted run does
    if space == "fermions_2s70":
        v = orc.coulomb_pseudopotentials(70)
        v[0::2] = 0.0
        sp = gpu.FermionOnSphereLong(4, 0, 70)
        H = gpu.ParticleOnSphereGenericHamiltonian(sp, 4, 70, v)
    else:
        v = orc.coulomb_pseudopotentials(45)
        v[1::2] = 0.0
        sp = gpu.BosonOnSphereShort(4, 2, 45)
        H = gpu.ParticleOnSphereGenericHamiltonian(sp, 4, 45, v)
    x0 = orc.random_vector(7, H.dim)
    a = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 600)
    a.InitializeLanczosAlgorithm(x0)
    ra = a.solve(max_iter=600)
    psi_a = a.GetGroundState()
    b = _lanczos(gpu, "ground", H, tmp_path, interval=4, max_iter=600)
    b.InitializeLanczosAlgorithm(x0)
    rb = b.solve(max_iter=21)
    assert not rb["converged"]
    del b
    c = _lanczos(gpu, "ground", H, tmp_path, max_iter=600)
    c.ResumeLanczosAlgorithm()
    rc = c.solve(max_iter=600)
    assert rc["converged"] and rb["iterations"] + rc["iterations"] == ra["iterations"]
    e = ra["eigenvalues"][0]
    assert abs(rc["eigenvalues"][0] - e) <= 1e-13 * abs(e)
    assert _overlap_error(c.GetGroundState(), psi_a) < 1e-10
