"""Generates the golden fixtures of the parity tests by running the reference itself.

Every fixture in this directory is produced by oracle/_ref/ref_tool (the reference compiled from
its own sources by `make -C oracle ref`; see oracle/ref_harness/ref_tool.cc for what each command
calls).  This script needs the reference checkout (default /root/reference, or $DIAGHAM_REF) and is
run by hand; the tests only read the .npz files it writes.

    python tests/golden/make_golden.py            # all small fixtures (about a minute)
    python tests/golden/make_golden.py --slow     # adds the long runs: the N=12, 2S=33 reference Lanczos
                                                  # and full product, the 91 sectors of N=10, 2S=27

Binary layouts written by ref_tool are documented next to each reader below.  Start vectors are
the repository's splitmix64 vectors (component i = (i+1)-th splitmix64 output of the seed mapped to
[-1, 1), normalised), written in DiagHam's vector format (int32 dimension + little-endian doubles,
RealVector::WriteVector, src/Vector/RealVector.cc:3669).
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TOOL = os.path.join(ROOT, "oracle", "_ref", "ref_tool")


def splitmix_vector(seed, dim):
    i = np.arange(1, dim + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    x = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0
    return x / np.sqrt(np.dot(x, x))


def uniform(seed, n, lo, hi):
    """n values uniform in [lo, hi) from splitmix64(seed), the same stream as splitmix_vector."""
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return lo + (hi - lo) * (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def write_vector(path, x):
    with open(path, "wb") as f:
        f.write(np.int32(len(x)).tobytes())
        f.write(np.ascontiguousarray(x, np.float64).tobytes())


def read_vector(path):
    b = open(path, "rb").read()
    d = int(np.frombuffer(b[:4], np.int32)[0])
    return np.frombuffer(b[4:4 + 8 * d], np.float64).copy()


def run(*args, env=None):
    cmd = [TOOL] + [str(a) for a in args]
    e = dict(os.environ)
    if env:
        e.update(env)
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, env=e)
    return " ".join(["ref_tool"] + [str(a) for a in args[:-1]])


def read_basis(path):
    # int64 dim, dim uint64 words, dim int32 lzmax (fermions only), dim int32 FindStateIndex
    b = open(path, "rb").read()
    d = int(np.frombuffer(b[:8], np.int64)[0])
    w = np.frombuffer(b[8:8 + 8 * d], np.uint64).copy()
    rest = np.frombuffer(b[8 + 8 * d:], np.int32).copy()
    return d, w, rest


def read_factors(path):
    # int32 nbrM12, per pair int32 (m1, m2, nbrM3, m3...), int32 nbrFactors, doubles
    b = np.fromfile(path, np.int32)
    p = int(b[0])
    i = 1
    m1, m2, nm3, m3 = [], [], [], []
    for _ in range(p):
        m1.append(b[i]); m2.append(b[i + 1]); nm3.append(b[i + 2])
        m3.extend(b[i + 3:i + 3 + b[i + 2]])
        i += 3 + b[i + 2]
    nf = int(b[i])
    fac = np.frombuffer(b[i + 1:].tobytes(), np.float64)[:nf].copy()
    return dict(m1=np.array(m1, np.int32), m2=np.array(m2, np.int32), nbr_m3=np.array(nm3, np.int32),
                m3=np.array(m3, np.int32), factors=fac)


def read_lanczos(path):
    # int32 nev, int32 iterations, int32 converged, double seconds, nev doubles, int32 nhist, nhist doubles
    b = open(path, "rb").read()
    nev, it, conv = np.frombuffer(b[:12], np.int32)
    eig = np.frombuffer(b[20:20 + 8 * nev], np.float64).copy()
    o = 20 + 8 * nev
    nh = int(np.frombuffer(b[o:o + 4], np.int32)[0])
    hist = np.frombuffer(b[o + 4:o + 4 + 8 * nh], np.float64).copy()
    return dict(nev=int(nev), iterations=int(it), converged=int(conv), eigenvalues=eig, history=hist)


def read_rows(path):
    # per row: int32 row, int32 count, count x (int32 target, int32 sign, int32 factor)
    b = np.fromfile(path, np.int32)
    i = 0
    rows, offs, trip = [], [0], []
    while i < len(b):
        r, c = b[i], b[i + 1]
        rows.append(r)
        trip.append(b[i + 2:i + 2 + 3 * c].reshape(c, 3))
        offs.append(offs[-1] + c)
        i += 2 + 3 * c
    t = np.concatenate(trip) if trip else np.zeros((0, 3), np.int32)
    return dict(rows=np.array(rows, np.int32), offsets=np.array(offs, np.int64), targets=t[:, 0].copy(),
                signs=t[:, 1].copy(), factor_index=t[:, 2].copy())


def coulomb_odd(two_s, tmp):
    p = os.path.join(tmp, "pp.bin")
    run("pseudopotentials", two_s, p)
    v = np.fromfile(p, np.float64)
    v[0::2] = 0.0
    return v


def save(name, cmd, **arrays):
    np.savez_compressed(os.path.join(HERE, name), command=np.array(cmd), **arrays)
    print("wrote", name)


def fermion_fixtures(tmp):
    for (n, s, lz) in [(4, 8, 2), (8, 21, 0), (5, 13, 1), (6, 15, 8), (3, 9, -3), (7, 18, 4)]:
        p = os.path.join(tmp, "b.bin")
        cmd = run("fqhe_basis", n, s, lz, p)
        d, w, rest = read_basis(p)
        save("fqhe_basis_n%d_2s%d_lz%d.npz" % (n, s, lz), cmd, words=w, lzmax=rest[:d], find=rest[d:2 * d])
    for s in (8, 21, 27, 33):
        p = os.path.join(tmp, "v.bin")
        cmd = run("pseudopotentials", s, p)
        save("pseudopotentials_2s%d.npz" % s, cmd, v=np.fromfile(p, np.float64))
    for (s, kind) in [(21, "v1"), (27, "coulomb"), (33, "coulomb")]:
        if kind == "v1":
            v = np.zeros(s + 1)
            v[1] = 1.0
        else:
            v = coulomb_odd(s, tmp)
        vf = os.path.join(tmp, "vv.bin")
        v.tofile(vf)
        p = os.path.join(tmp, "f.bin")
        cmd = run("fqhe_factors", 8, s, vf, p)
        save("factors_2s%d_%s.npz" % (s, kind), cmd, v=v, **read_factors(p))


def fqhe_sector_fixtures(tmp, n, s, lz, kind, rows_sample, lanczos=True, algos=("basic",)):
    if kind == "v1":
        v = np.zeros(s + 1)
        v[1] = 1.0
    else:
        v = coulomb_odd(s, tmp)
    vf = os.path.join(tmp, "vv.bin")
    v.tofile(vf)
    tag = "n%d_2s%d_lz%d_%s" % (n, s, lz, kind)
    rows = np.asarray(rows_sample, np.int32)
    rf = os.path.join(tmp, "rows.bin")
    rows.tofile(rf)
    p = os.path.join(tmp, "rows.out")
    cmd = run("fqhe_rows", n, s, lz, vf, rf, p)
    save("rows_%s.npz" % tag, cmd, v=v, **read_rows(p))
    if not lanczos:
        return
    from math import comb  # noqa: F401  (dimension comes from the basis fixture / oracle)
    dfile = os.path.join(tmp, "b.bin")
    run("fqhe_basis", n, s, lz, dfile)
    dim, _, _ = read_basis(dfile)
    x = splitmix_vector(0, dim)
    xf = os.path.join(tmp, "x0.vec")
    write_vector(xf, x)
    for shift in (0.0, 0.37):
        yf = os.path.join(tmp, "y.vec")
        cmd = run("fqhe_matvec", n, s, lz, vf, xf, shift, yf)
        save("matvec_%s_shift%g.npz" % (tag, shift), cmd, v=v, seed=0, shift=shift, y=read_vector(yf))
    for algo in algos:
        lf = os.path.join(tmp, "l.out")
        gf = os.path.join(tmp, "gs.vec")
        cmd = run("fqhe_lanczos", n, s, lz, vf, algo, 1, 1, 200, 0, lf, gf if algo == "ground" else "-", xf)
        extra = {}
        if algo == "ground":
            psi = read_vector(gf)
            ef = os.path.join(tmp, "expect.bin")
            run("fqhe_expect", n, s, lz, vf, gf, ef)
            e = np.fromfile(ef, np.float64)
            extra = dict(expectation=e[:-1], energy_expectation=e[-1], psi_norm=np.linalg.norm(psi))
        save("lanczos_%s_%s.npz" % (tag, algo), cmd, v=v, seed=0, max_iter=200, **read_lanczos(lf), **extra)


def block_fixture(tmp, n, s, lz, k):
    v = coulomb_odd(s, tmp)
    vf = os.path.join(tmp, "vv.bin")
    v.tofile(vf)
    dfile = os.path.join(tmp, "b.bin")
    run("fqhe_basis", n, s, lz, dfile)
    dim, _, _ = read_basis(dfile)
    # BasicBlockLanczosAlgorithm uses given start vectors as they are (InitializeLanczosAlgorithm,
    # BasicBlockLanczosAlgorithm.cc:262-300), so the block is orthonormalised here first
    block, _ = np.linalg.qr(np.stack([splitmix_vector(100 + b, dim) for b in range(k)], axis=1))
    files = []
    for b in range(k):
        xf = os.path.join(tmp, "xb%d.vec" % b)
        write_vector(xf, block[:, b])
        files.append(xf)
    lf = os.path.join(tmp, "l.out")
    cmd = run("fqhe_lanczos", n, s, lz, vf, "block", 2, k, 400, 0, lf, "-", *files)
    save("lanczos_n%d_2s%d_lz%d_coulomb_block%d.npz" % (n, s, lz, k), cmd, v=v, seeds=np.arange(100, 100 + k),
         **read_lanczos(lf))


def spin_fixtures(tmp):
    for (L, sz) in [(10, 0), (9, 1), (12, 0), (12, -4), (32, 30)]:
        p = os.path.join(tmp, "sb.bin")
        cmd = run("spin_basis", L, sz, p)
        d, w, rest = read_basis(p)
        save("spin_basis_L%d_sz%d.npz" % (L, sz), cmd, words=w, find=rest[:d])
    for (L, sz, j1, j2) in [(12, 0, 1.0, 0.5), (11, 1, 1.0, 0.3), (10, 2, 0.7, -0.4)]:
        p = os.path.join(tmp, "sb.bin")
        run("spin_basis", L, sz, p)
        d, _, _ = read_basis(p)
        xf = os.path.join(tmp, "sx.vec")
        write_vector(xf, splitmix_vector(3, d))
        yf = os.path.join(tmp, "sy.vec")
        cmd = run("spin_matvec", L, sz, j1, j2, xf, yf)
        save("spin_matvec_L%d_sz%d_j%g_%g.npz" % (L, sz, j1, j2), cmd, seed=3, y=read_vector(yf))
    for (L, sz, j1, j2) in [(16, 0, 1.0, 0.5), (14, 0, 1.0, 0.2), (13, 1, 1.0, 0.5)]:
        p = os.path.join(tmp, "sb.bin")
        run("spin_basis", L, sz, p)
        d, _, _ = read_basis(p)
        xf = os.path.join(tmp, "sx.vec")
        write_vector(xf, splitmix_vector(0, d))
        lf = os.path.join(tmp, "sl.out")
        cmd = run("spin_lanczos", L, sz, j1, j2, "basic", 1, 1, 400, 0, lf, xf)
        save("spin_lanczos_L%d_sz%d_j%g_%g.npz" % (L, sz, j1, j2), cmd, seed=0, **read_lanczos(lf))


def slow_fixtures(tmp):
    # the precision workload: N = 12, 2S = 33, Lz = 0, LLL Coulomb (odd m), start vector seed 0
    v = coulomb_odd(33, tmp)
    vf = os.path.join(tmp, "vv.bin")
    v.tofile(vf)
    dim = 7764392
    xf = os.path.join(tmp, "x0.vec")
    write_vector(xf, splitmix_vector(0, dim))
    lf = os.path.join(tmp, "l.out")
    threads = os.cpu_count() or 1
    cmd = run("fqhe_lanczos", 12, 33, 0, vf, "basic", 1, 1, 400, 1e-13, lf, "-", xf, env={"REF_THREADS": str(threads)})
    save("lanczos_n12_2s33_lz0_coulomb_basic.npz", cmd + " (REF_THREADS=%d)" % threads, v=v, seed=0, precision=1e-13,
         **read_lanczos(lf))


def read_sectors(path):
    # text, one line per sector: 2Lz dim E0 iterations converged method
    rows = [l.split() for l in open(path) if l.strip()]
    rows.sort(key=lambda r: int(r[0]))
    return dict(two_lz=np.array([int(r[0]) for r in rows], np.int32), dims=np.array([int(r[1]) for r in rows], np.int64),
                e0=np.array([float(r[2]) for r in rows]), iterations=np.array([int(r[3]) for r in rows], np.int32),
                converged=np.array([int(r[4]) for r in rows], np.int32),
                method=np.array([r[5] for r in rows]))


def sectors_fixture(tmp, out=None):
    # the batching workload: N = 10, 2S = 27, every sector 2Lz = 0..180, V_1 = 1 and V_3, V_5, V_7
    # uniform in [0, 0.5) from splitmix64 seed 1; the reference's block Lanczos (k = 4, its own random
    # start, stopping at 1e-13) per sector, full diagonalisation below 300 states (about 15 minutes
    # on 8 threads)
    v = np.zeros(28)
    v[1] = 1.0
    v[[3, 5, 7]] = uniform(1, 3, 0.0, 0.5)
    vf = os.path.join(tmp, "v27.bin")
    v.tofile(vf)
    out = out or os.path.join(tmp, "sectors.txt")
    threads = os.cpu_count() or 1
    cmd = run("fqhe_sectors", 10, 27, vf, 4, 2000, 1e-13, 300, out, env={"REF_THREADS": str(threads)})
    save("sectors_n10_2s27_block4.npz", cmd + " (REF_THREADS=%d)" % threads, v=v, block=4, precision=1e-13,
         full_diag=300, **read_sectors(out))


def product_fixture_n12_2s33(tmp):
    # the precision workload's full product: y = H x for the splitmix64 seed-5 vector, computed by the
    # reference's SMP product (non-hermitian LowLevelMultiply split over threads); 62 MB, so only a
    # strided sample of y (every 997th entry), its norm and its dot products with two more seeded
    # vectors are kept (about a minute on 8 threads)
    v = coulomb_odd(33, tmp)
    vf = os.path.join(tmp, "vv.bin")
    v.tofile(vf)
    dim = 7764392
    xf = os.path.join(tmp, "x5.vec")
    write_vector(xf, splitmix_vector(5, dim))
    yf = os.path.join(tmp, "y5.vec")
    threads = os.cpu_count() or 1
    cmd = run("fqhe_matvec", 12, 33, 0, vf, xf, 0.0, yf, env={"REF_THREADS": str(threads)})
    y = read_vector(yf)
    stride = 997
    save("product_n12_2s33_lz0_coulomb_seed5.npz", cmd + " (REF_THREADS=%d)" % threads, v=v, seed=5, stride=stride,
         sample=y[::stride].copy(), norm=np.linalg.norm(y), max_abs=np.max(np.abs(y)),
         dot_seed6=float(np.dot(y, splitmix_vector(6, dim))), dot_seed7=float(np.dot(y, splitmix_vector(7, dim))),
         x_dot_y=float(np.dot(y, splitmix_vector(5, dim))))


def gradient_fixtures(tmp):
    # the differentiation workload: N = 10, 2S = 27, 2Lz = 0 and 2 (Lz = 0, 1); LLL Coulomb V_m
    # (every m) plus uniform [-0.05, 0.05) noise from splitmix64 seed 2.  The reference's
    # BasicLanczosAlgorithmWithGroundState (precision 1e-14, start vector seed 0) gives E0 and psi;
    # ParticleOnSphereGenericHamiltonian(V = e_m).MatrixElement(psi, psi) for every m is the FP64
    # reference gradient dE0/dV_m (Hellmann-Feynman; the interaction factors are linear in V)
    p = os.path.join(tmp, "pp.bin")
    run("pseudopotentials", 27, p)
    v = np.fromfile(p, np.float64) + uniform(2, 28, -0.05, 0.05)
    vf = os.path.join(tmp, "vg.bin")
    v.tofile(vf)
    threads = os.cpu_count() or 1
    for lz in (0, 2):
        bf = os.path.join(tmp, "b.bin")
        run("fqhe_basis", 10, 27, lz, bf)
        dim, _, _ = read_basis(bf)
        xf = os.path.join(tmp, "xg.vec")
        write_vector(xf, splitmix_vector(0, dim))
        lf, gf, ef = (os.path.join(tmp, n) for n in ("lg.out", "gg.vec", "eg.bin"))
        cmd = run("fqhe_lanczos", 10, 27, lz, vf, "ground", 1, 1, 600, 1e-14, lf, gf, xf,
                  env={"REF_THREADS": str(threads)})
        run("fqhe_expect", 10, 27, lz, vf, gf, ef)
        e = np.fromfile(ef, np.float64)
        save("gradient_n10_2s27_lz%d.npz" % lz, cmd + " (REF_THREADS=%d)" % threads, v=v, seed=0, precision=1e-14,
             dim=dim, expectation=e[:-1], energy_expectation=e[-1], **read_lanczos(lf))


def l2_fixtures(tmp):
    # y = L^2 x by the reference's ParticleOnSphereL2Hamiltonian (l2Factor 1, fixed Lz, on the fly,
    # hermitian symmetry off) for x = the splitmix64 vector of seed 7
    for (n, s, lz) in [(6, 15, 0), (6, 15, 4), (7, 18, 2), (8, 21, 0), (8, 21, 6)]:
        bf = os.path.join(tmp, "b.bin")
        run("fqhe_basis", n, s, lz, bf)
        dim, _, _ = read_basis(bf)
        xf, yf = os.path.join(tmp, "xl2.vec"), os.path.join(tmp, "yl2.vec")
        write_vector(xf, splitmix_vector(7, dim))
        cmd = run("fqhe_l2", n, s, lz, xf, yf)
        save("l2_n%d_2s%d_lz%d.npz" % (n, s, lz), cmd, seed=7, y=read_vector(yf))
    # the same product on BosonOnSphereShort sectors (the operator's bosonic branch)
    for (n, s, lz) in [(6, 10, 0), (5, 9, 1), (7, 12, 2), (8, 14, 0), (8, 8, 4)]:
        bf = os.path.join(tmp, "bb.bin")
        run("bqhe_basis", n, s, lz, bf)
        dim = int(np.frombuffer(open(bf, "rb").read(8), np.int64)[0])
        xf, yf = os.path.join(tmp, "xl2.vec"), os.path.join(tmp, "yl2.vec")
        write_vector(xf, splitmix_vector(7, dim))
        cmd = run("bqhe_l2", n, s, lz, xf, yf)
        save("boson_l2_n%d_2s%d_lz%d.npz" % (n, s, lz), cmd, seed=7, y=read_vector(yf))


def boson_fixtures(tmp):
    # BosonOnSphereShort with ParticleOnSphereGenericHamiltonian (on the fly, hermitian symmetry off):
    # the basis as occupations (PrintState), y = H x for x = the splitmix64 vector of seed 0 (shift 0
    # and 0.37), and the basic Lanczos run from that vector (precision MACHINE_PRECISION, 300 iterations
    # at most).  "coulomb" = the LLL Coulomb V_m with the odd m set to zero, "v0" = the delta interaction.
    for (n, s, lz, kind) in [(4, 6, 0, "v0"), (6, 10, 0, "v0"), (6, 10, 0, "coulomb"), (5, 9, 1, "coulomb"),
                             (7, 12, 2, "coulomb"), (8, 8, 0, "coulomb"), (8, 14, 0, "coulomb")]:
        p = os.path.join(tmp, "pp.bin")
        run("pseudopotentials", s, p)
        v = np.fromfile(p, np.float64)
        v[1::2] = 0.0
        if kind == "v0":
            v = np.zeros(s + 1)
            v[0] = 1.0
        vf = os.path.join(tmp, "vb.bin")
        v.tofile(vf)
        bf = os.path.join(tmp, "bb.bin")
        cmd = run("bqhe_basis", n, s, lz, bf)
        b = open(bf, "rb").read()
        dim = int(np.frombuffer(b[:8], np.int64)[0])
        occ = np.frombuffer(b[8:], np.int32).reshape(dim, s + 1).copy()
        xf = os.path.join(tmp, "xb.vec")
        write_vector(xf, splitmix_vector(0, dim))
        ys = {}
        for shift in (0.0, 0.37):
            yf = os.path.join(tmp, "yb.vec")
            cmd2 = run("bqhe_matvec", n, s, lz, vf, xf, shift, yf)
            ys["y_shift%g" % shift] = read_vector(yf)
        lf = os.path.join(tmp, "lb.out")
        cmd3 = run("bqhe_lanczos", n, s, lz, vf, "basic", 1, 1, 300, 0, lf, "-", xf)
        save("boson_n%d_2s%d_lz%d_%s.npz" % (n, s, lz, kind), "; ".join([cmd, cmd2, cmd3]), v=v, seed=0,
             occupations=occ, max_iter=300, **ys, **read_lanczos(lf))


BOSON_LARGE_CASES = [(2, 61, 0), (3, 40, 0), (3, 60, 0), (4, 45, 2), (5, 50, 0)]


def boson_large_fixtures(tmp):
    # BosonOnSphereShort beyond 41-bit words (lz_max + N - 1 = 42 to 62, the reference's own range for
    # this class): the states as their fermionic words (n_0 ones, a zero, n_1 ones, ...), or the SHA-256 of
    # those words above 13,000 states, y = H x (x = splitmix64 seed 0) at shifts 0 and 0.37 (shift 0 only
    # above 13,000 states) from the reference's product with the exact interaction factors written into
    # its table (bqhe_matvec_f; its own factors drift at this 2S, so its own product is kept beside it
    # with the factors' deviation), and the basic Lanczos run (its own factors) where the sector has at
    # most 13,000 states; V = the reference's own LLL Coulomb pseudopotentials with the odd m set to zero
    import hashlib
    for (n, s, lz) in BOSON_LARGE_CASES:
        p = os.path.join(tmp, "pp.bin")
        run("pseudopotentials", s, p)
        v = np.fromfile(p, np.float64)
        v[1::2] = 0.0
        vf = os.path.join(tmp, "vb.bin")
        v.tofile(vf)
        bf = os.path.join(tmp, "bb.bin")
        cmd = run("bqhe_basis", n, s, lz, bf)
        b = open(bf, "rb").read()
        dim = int(np.frombuffer(b[:8], np.int64)[0])
        occ = np.frombuffer(b[8:], np.int32).reshape(dim, s + 1)
        words = np.zeros(dim, np.uint64)
        for i in range(dim):
            w, pos = 0, 0
            for m in range(s + 1):
                w |= ((1 << int(occ[i, m])) - 1) << pos
                pos += int(occ[i, m]) + 1
            words[i] = w
        xf = os.path.join(tmp, "xb.vec")
        write_vector(xf, splitmix_vector(0, dim))
        exact, own = exact_factors_in_reference_order(tmp, n, s, v, bosons=True)
        ff = os.path.join(tmp, "fb.bin")
        exact.tofile(ff)
        ys = {"own_factor_deviation": np.max(np.abs(exact - own)) / np.max(np.abs(exact))}
        for shift in ((0.0, 0.37) if dim <= 13000 else (0.0,)):
            yf = os.path.join(tmp, "yb.vec")
            run("bqhe_matvec", n, s, lz, vf, xf, shift, yf)
            ys["y_own_factors_shift%g" % shift] = read_vector(yf)
            cmd2 = run("bqhe_matvec_f", n, s, lz, vf, ff, xf, shift, yf)
            ys["y_shift%g" % shift] = read_vector(yf)
        extra = {}
        if dim <= 13000:
            lf = os.path.join(tmp, "lb.out")
            run("bqhe_lanczos", n, s, lz, vf, "basic", 1, 1, 300, 0, lf, "-", xf)
            extra = read_lanczos(lf)
            extra["words"] = words
        else:
            extra["words_sha256"] = hashlib.sha256(words.tobytes()).hexdigest()
        save("boson_large_n%d_2s%d_lz%d.npz" % (n, s, lz), cmd + "; " + cmd2, v=v, seed=0, dim=dim, **ys, **extra)


ENTANGLEMENT_CASES = [(11, 4, 0), (11, 4, 2), (11, 3, -3), (5, 2, 0), (1, 1, 0), (1, 0, 0), (0, 0, 0), (11, 0, 0),
                      (21, 8, 0), (15, 8, 56), (20, 7, -5), (22, 8, 0)]


def entanglement_fixtures(tmp):
    # FermionOnSphere::EvaluatePartialEntanglementMatrix / EvaluatePartialDensityMatrix (orbital cut l,
    # nbrFermionSector NA, lzSector 2LzA) of x = the splitmix64 vector of seed 0 on N=8 2S=21 2Lz=0;
    # rho is stored for the cases with at most 600 rows (M M^T is checked against it)
    def rd(path):
        b = open(path, "rb").read()
        r, c = np.frombuffer(b[:16], np.int64)
        return np.frombuffer(b[16:], np.float64).reshape(r, c).copy()
    n, s, lz = 8, 21, 0
    bf = os.path.join(tmp, "b.bin")
    run("fqhe_basis", n, s, lz, bf)
    dim, _, _ = read_basis(bf)
    xf = os.path.join(tmp, "xe.vec")
    write_vector(xf, splitmix_vector(0, dim))
    out, cmds = {}, []
    for (l, na, lza) in ENTANGLEMENT_CASES:
        tag = "l%d_na%d_lz%d" % (l, na, lza)
        ef, df = os.path.join(tmp, "e.bin"), os.path.join(tmp, "d.bin")
        cmds.append(run("fqhe_entanglement", n, s, lz, xf, l, na, lza, ef))
        out["m_" + tag] = rd(ef)
        if l <= s and out["m_" + tag].shape[0] <= 600:
            run("fqhe_density", n, s, lz, xf, l, na, lza, df)
            out["rho_" + tag] = rd(df)
    save("entanglement_n%d_2s%d_lz%d.npz" % (n, s, lz), cmds[0] + " (and fqhe_density, per case)", seed=0,
         cases=np.array(ENTANGLEMENT_CASES, np.int32), **out)


TRANSLATION_CASES = [(8, 0, 0, 1.0, 0.5), (8, 0, 4, 1.0, 0.5), (12, 0, 0, 1.0, 0.5), (12, 0, 6, 1.0, 0.3),
                     (12, 2, 6, 1.0, 0.5), (13, 1, 0, 1.0, 0.3), (16, 0, 0, 1.0, 0.5), (16, 0, 8, 1.0, 0.2),
                     (18, 2, 0, 1.0, 0.5), (20, 0, 10, 1.0, 0.4)]


def translation_fixtures(tmp):
    # Spin1_2ChainWithTranslations(L, K, 1, 2Sz) with SpinChainJ1J2RealHamiltonianWithTranslations(J1, J2):
    # the representatives (ascending), y = H x for x = the splitmix64 vector of seed 0, and the basic
    # Lanczos run from it (precision MACHINE_PRECISION, 300 iterations at most) where the sector has
    # 300 states or more (below that the reference's run outlives the Krylov space)
    for (L, sz, k, j1, j2) in TRANSLATION_CASES:
        bf = os.path.join(tmp, "tb.bin")
        cmd = run("spint_basis", L, sz, k, bf)
        b = open(bf, "rb").read()
        dim = int(np.frombuffer(b[:8], np.int64)[0])
        words = np.frombuffer(b[8:], np.uint64).copy()
        xf = os.path.join(tmp, "xt.vec")
        write_vector(xf, splitmix_vector(0, dim))
        yf = os.path.join(tmp, "yt.vec")
        cmd2 = run("spint_matvec", L, sz, k, j1, j2, xf, yf)
        extra = {}
        if dim >= 300:
            lf = os.path.join(tmp, "lt.out")
            run("spint_lanczos", L, sz, k, j1, j2, 300, 0, lf, xf)
            extra = read_lanczos(lf)
        save("translations_L%d_sz%d_k%d_j2_%g.npz" % (L, sz, k, j2), cmd + "; " + cmd2, seed=0, j1=j1, j2=j2,
             words=words, y=read_vector(yf), **extra)


LONG_CASES = [  # (space, N, 2S, 2Lz): FermionOnSphere beyond 2S = 40 and FermionOnSphereLong
    ("fermion", 3, 62, 0), ("fermion", 4, 50, 0), ("fermion", 5, 41, 1),
    ("long", 2, 126, -2), ("long", 3, 63, 1), ("long", 3, 126, 0), ("long", 4, 70, 0), ("long", 4, 100, 2),
    ("long", 5, 64, 0)]


def coulomb_closed_form(two_s):
    """LLL Coulomb pseudopotentials on the sphere from the closed form (Fano, Ortolani and Colombo):
    V_m = 2 / sqrt(S) C(4S - 2L, 2S - L) C(4S + 2L + 2, 2S + L + 1) / C(4S + 2, 2S + 1)^2, L = 2S - m,
    evaluated in exact integer arithmetic and rounded once."""
    from fractions import Fraction
    from math import comb, sqrt
    out = np.zeros(two_s + 1)
    for m in range(two_s + 1):
        L = two_s - m
        f = Fraction(2 * comb(2 * two_s - 2 * L, two_s - L) * comb(2 * two_s + 2 * L + 2, two_s + L + 1),
                     comb(2 * two_s + 2, two_s + 1) ** 2)
        out[m] = float(f) / sqrt(two_s / 2)
    return out


def exact_factors_in_reference_order(tmp, n, s, v, bosons=False):
    """The oracle's interaction factors (Clebsch-Gordan coefficients exact to the last bit) laid out in
    the reference's own (pair, m3) order, read from its lfqhe_factors (bqhe_factors) table."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    vf = os.path.join(tmp, "vf.bin")
    v.tofile(vf)
    ff = os.path.join(tmp, "ff.bin")
    run("bqhe_factors" if bosons else "lfqhe_factors", n, s, vf, ff)
    r = read_factors(ff)
    t = oracle.boson_interaction_tables(s, v) if bosons else oracle.interaction_tables(s, v)
    ours = {}
    for p in range(len(t["m1"])):
        o = int(t["m3_offset"][p])
        for q in range(int(t["nbr_m3"][p])):
            ours[(int(t["m1"][p]), int(t["m2"][p]), int(t["m3"][o + q]))] = float(t["factors"][o + q])
    out, off = [], 0
    for p in range(len(r["m1"])):
        for q in range(int(r["nbr_m3"][p])):
            out.append(ours[(int(r["m1"][p]), int(r["m2"][p]), int(r["m3"][off + q]))])
        off += int(r["nbr_m3"][p])
    return np.array(out), r["factors"]


def long_fixtures(tmp):
    # the words ((low, high) uint64 pairs), y = H x at shifts 0 and 0.37 for x = the splitmix64 vector of
    # seed 0, and the basic Lanczos run from it (sectors up to 13,000 states), with V = the closed-form
    # Coulomb pseudopotentials (odd m; both sides take the same file, so the products do not depend on
    # either code's pseudopotential routine).  The reference's own interaction factors drift from the
    # exact ones as 2S grows (3.6e-13 at 2S = 62, 1.4e-12 at 70, 33% at 100, 87% at 126: its
    # Clebsch-Gordan evaluation), so for FermionOnSphereLong y is the reference's product with the exact
    # factors put in its tables (lfqhe_matvec_f), and its product with its own factors is kept beside it
    # (y_own_factors_*) with the factors' largest deviation; its Lanczos is recorded only up to 2S = 84.
    # Also the reference's own EvaluatePseudopotentials at large 2S next to the closed form.
    for (space, n, s, lz) in LONG_CASES:
        prefix = "fqhe" if space == "fermion" else "lfqhe"
        v = coulomb_closed_form(s)
        v[0::2] = 0.0
        vf = os.path.join(tmp, "vl.bin")
        v.tofile(vf)
        bf = os.path.join(tmp, "bl.bin")
        cmd = run(prefix + "_basis", n, s, lz, bf)
        if space == "fermion":
            dim, w, _ = read_basis(bf)
            words = np.stack([w, np.zeros_like(w)], axis=1)
        else:
            b = open(bf, "rb").read()
            dim = int(np.frombuffer(b[:8], np.int64)[0])
            words = np.frombuffer(b[8:8 + 16 * dim], np.uint64).reshape(dim, 2).copy()
        xf = os.path.join(tmp, "xl.vec")
        write_vector(xf, splitmix_vector(0, dim))
        ys = {}
        if space == "long":
            exact, own = exact_factors_in_reference_order(tmp, n, s, v)
            ff = os.path.join(tmp, "fe.bin")
            exact.tofile(ff)
            ys["own_factor_deviation"] = np.max(np.abs(exact - own)) / np.max(np.abs(exact))
        for shift in (0.0, 0.37):
            yf = os.path.join(tmp, "yl.vec")
            cmd2 = run(prefix + "_matvec", n, s, lz, vf, xf, shift, yf)
            if space == "long":
                ys["y_own_factors_shift%g" % shift] = read_vector(yf)
                cmd2 = run("lfqhe_matvec_f", n, s, lz, vf, ff, xf, shift, yf)
            ys["y_shift%g" % shift] = read_vector(yf)
        extra = {}
        if dim <= 13000 and s <= 84:
            lf = os.path.join(tmp, "ll.out")
            run(prefix + "_lanczos", n, s, lz, vf, "basic", 1, 1, 300, 0, lf, "-", xf)
            extra = read_lanczos(lf)
        if dim > 13000:
            # large sectors: the words as a SHA-256 of their (low, high) bytes, y at shift 0 only
            import hashlib
            ys = {"y_shift0": ys["y_shift0"], "own_factor_deviation": ys.get("own_factor_deviation", 0.0)}
            save("long_%s_n%d_2s%d_lz%d.npz" % (space, n, s, lz), cmd + "; " + cmd2, v=v, seed=0, dim=dim,
                 words_sha256=hashlib.sha256(words.tobytes()).hexdigest(), **ys, **extra)
            continue
        save("long_%s_n%d_2s%d_lz%d.npz" % (space, n, s, lz), cmd + "; " + cmd2, v=v, seed=0, words=words,
             **ys, **extra)
    sizes = np.array([84, 100, 126])
    ref = {}
    for s in sizes:
        pf = os.path.join(tmp, "pl.bin")
        run("pseudopotentials", s, pf)
        ref["reference_%d" % s] = np.fromfile(pf, np.float64)[-(s + 1):]
        ref["closed_form_%d" % s] = coulomb_closed_form(int(s))
    save("pseudopotentials_large_2s.npz", "ref_tool pseudopotentials 2S", sizes=sizes, **ref)


TRANSLATION_COMPLEX_CASES = [(8, 0, 1, 1.0, 0.5), (8, 0, 3, 1.0, 0.3), (12, 0, 2, 1.0, 0.5), (12, 2, 5, 1.0, 0.4),
                             (13, 1, 3, 1.0, 0.3), (16, 0, 3, 1.0, 0.2), (18, 0, 4, 1.0, 0.5), (20, 2, 7, 1.0, 0.3)]


def write_complex_vector(path, z):
    # ComplexVector::WriteVector: int32 dimension, then (Re, Im) pairs as doubles
    with open(path, "wb") as f:
        f.write(np.int32(len(z)).tobytes())
        f.write(np.ascontiguousarray(np.stack([z.real, z.imag], axis=1)).tobytes())


def read_complex_vector(path):
    b = open(path, "rb").read()
    d = int(np.frombuffer(b[:4], np.int32)[0])
    a = np.frombuffer(b[4:4 + 16 * d], np.float64).reshape(d, 2)
    return a[:, 0] + 1j * a[:, 1]


def translation_complex_fixtures(tmp):
    # SpinChainJ1J2HamiltonianWithTranslations (complex, any K) on Spin1_2ChainWithTranslations(L, K, 1,
    # 2Sz): y = H x for x = (splitmix64 seed 0) + i (splitmix64 seed 1), and, for sectors up to 900
    # states, the reference's dense matrix (assembled column by column through its own product)
    # diagonalised by LAPACK: its four lowest eigenvalues and how far it is from Hermitian
    for (L, sz, k, j1, j2) in TRANSLATION_COMPLEX_CASES:
        bf = os.path.join(tmp, "tcb.bin")
        run("spint_basis", L, sz, k, bf)
        b = open(bf, "rb").read()
        dim = int(np.frombuffer(b[:8], np.int64)[0])
        words = np.frombuffer(b[8:], np.uint64).copy()
        x = splitmix_vector(0, dim) + 1j * splitmix_vector(1, dim)
        xf = os.path.join(tmp, "tcx.vec")
        write_complex_vector(xf, x)
        yf = os.path.join(tmp, "tcy.vec")
        cmd = run("spintc_matvec", L, sz, k, j1, j2, xf, yf)
        extra = {}
        if dim <= 900:
            df = os.path.join(tmp, "tcd.bin")
            run("spintc_dense", L, sz, k, j1, j2, df)
            m = np.fromfile(df, np.float64, offset=8).reshape(dim, dim, 2)
            m = m[:, :, 0] + 1j * m[:, :, 1]
            extra = dict(hermitian_error=np.max(np.abs(m - m.conj().T)),
                         eigenvalues=np.linalg.eigvalsh(0.5 * (m + m.conj().T))[:4])
        save("translations_complex_L%d_sz%d_k%d_j2_%g.npz" % (L, sz, k, j2), cmd, seed_re=0, seed_im=1, j1=j1,
             j2=j2, words=words, y=read_complex_vector(yf), **extra)
        if (L, sz, k) == (8, 0, 1):
            # a file written by ComplexVector::WriteVector itself, for the vector-file tests
            import shutil
            shutil.copyfile(yf, os.path.join(HERE, "complexvector_translations_L8_sz0_k1.vec"))


def dir_files(d):
    names = sorted(os.listdir(d))
    return np.array(names), {"f%d" % i: np.frombuffer(open(os.path.join(d, f), "rb").read(), np.uint8)
                             for i, f in enumerate(names)}


def disk_fixtures(tmp):
    # The disk-storage Lanczos classes (BasicLanczosAlgorithmWithDiskStorage = "basic",
    # BasicLanczosAlgorithmWithGroundStateDiskStorage = "ground") on N=7 2S=18 2Lz=2, odd Coulomb
    # pseudopotentials, start = splitmix64 vector of seed 0, precision MACHINE_PRECISION:
    #   interrupted_*  the files of the run stopped at counter 14 (file names in interrupted_names,
    #                  contents as raw bytes in interrupted_f<i>)
    #   resumed        the driver loop resumed from those files (counter from 0)
    #   full           the uninterrupted run (and its ground state psi for "ground")
    #   assembly_*     ("ground") the files after the resumed run assembled its ground state for 5
    #                  steps only (GroundStateEvaluationFlag 1)
    import shutil
    n, s, lz, stop = 7, 18, 2, 14
    v = coulomb_odd(s, tmp)
    vf = os.path.join(tmp, "vv.bin")
    v.tofile(vf)
    bf = os.path.join(tmp, "b.bin")
    run("fqhe_basis", n, s, lz, bf)
    dim, _, _ = read_basis(bf)
    xf = os.path.join(tmp, "x0.vec")
    write_vector(xf, splitmix_vector(0, dim))
    lf = os.path.join(tmp, "l.out")
    for algo in ("basic", "ground"):
        d_full, d_int, d_res = (os.path.join(tmp, "%s_%s" % (algo, k)) for k in ("full", "int", "res"))
        for d in (d_full, d_int):
            os.makedirs(d)
        gf = os.path.join(tmp, "gs_full.vec")
        cmd = run("fqhe_lanczos_disk", n, s, lz, vf, algo, 400, 0, d_full, xf, 100000, lf,
                  gf if algo == "ground" else "-")
        full = read_lanczos(lf)
        cmd_int = run("fqhe_lanczos_disk", n, s, lz, vf, algo, stop, 0, d_int, xf, 100000, lf, "-")
        int_names, int_files = dir_files(d_int)
        shutil.copytree(d_int, d_res)
        cmd_res = run("fqhe_lanczos_disk", n, s, lz, vf, algo, 400, 0, d_res, "resume", 100000, lf, "-")
        res = read_lanczos(lf)
        extra = {}
        if algo == "ground":
            run("fqhe_lanczos_disk", n, s, lz, vf, algo, 400, 0, d_res, "resume", 5, lf, os.path.join(tmp, "gs5.vec"))
            a_names, a_files = dir_files(d_res)
            extra = dict(psi=read_vector(gf), assembly_names=a_names,
                         **{"assembly_" + k: b for k, b in a_files.items()})
        save("disk_%s_n%d_2s%d_lz%d.npz" % (algo, n, s, lz), "; ".join([cmd, cmd_int, cmd_res]), v=v, seed=0, stop=stop,
             full_iterations=full["iterations"], full_eigenvalue=full["eigenvalues"][0],
             resumed_iterations=res["iterations"], resumed_eigenvalue=res["eigenvalues"][0],
             interrupted_names=int_names, **{"interrupted_" + k: b for k, b in int_files.items()}, **extra)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--slow", action="store_true")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not os.path.exists(TOOL):
        sys.exit("build the reference first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        if args.only in (None, "fermion"):
            fermion_fixtures(tmp)
        if args.only in (None, "sectors"):
            fqhe_sector_fixtures(tmp, 8, 21, 0, "v1", [0, 1, 2, 77, 4000, 8511])
            fqhe_sector_fixtures(tmp, 8, 21, 0, "coulomb", [0, 5, 100, 2222, 8000, 8511],
                                 algos=("basic", "full", "ground"))
            fqhe_sector_fixtures(tmp, 7, 18, 2, "coulomb", [0, 3, 500, 1000], algos=("basic",))
            rng = np.random.default_rng(12)
            big = np.concatenate([[0, 1, 7764391], rng.integers(0, 7764392, 13)]).astype(np.int32)
            fqhe_sector_fixtures(tmp, 12, 33, 0, "coulomb", big, lanczos=False)
            mid = np.concatenate([[0, 246447], rng.integers(0, 246448, 10)]).astype(np.int32)
            fqhe_sector_fixtures(tmp, 10, 27, 0, "coulomb", mid, lanczos=False)
        if args.only in (None, "block"):
            block_fixture(tmp, 6, 15, 0, 4)
        if args.only in (None, "spin"):
            spin_fixtures(tmp)
        if args.only in (None, "gradient"):
            gradient_fixtures(tmp)
        if args.only in (None, "l2"):
            l2_fixtures(tmp)
        if args.only in (None, "disk"):
            disk_fixtures(tmp)
        if args.only in (None, "boson"):
            boson_fixtures(tmp)
        if args.only in (None, "entanglement"):
            entanglement_fixtures(tmp)
        if args.only in (None, "translations"):
            translation_fixtures(tmp)
        if args.only in (None, "long"):
            long_fixtures(tmp)
        if args.only in (None, "boson_large"):
            boson_large_fixtures(tmp)
        if args.only in (None, "translations_complex"):
            translation_complex_fixtures(tmp)
        if args.slow:
            slow_fixtures(tmp)
        if args.slow or args.only == "product_n12":
            product_fixture_n12_2s33(tmp)
        if args.slow or args.only == "sectors_n10":
            sectors_fixture(tmp)


if __name__ == "__main__":
    main()
