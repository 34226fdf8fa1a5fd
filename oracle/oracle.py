"""ctypes view of liboracle.so, the CPU restatement of DiagHam's H.v + Lanczos path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, and there only as the checker.  The product
package (diagham_b200) never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_f64p = ctypes.POINTER(ctypes.c_double)


def build():
    """Compile liboracle.so in place (plain gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        L.orc_fermion_dimension.restype = ctypes.c_long
        L.orc_fermion_dimension.argtypes = [ctypes.c_int] * 3
        L.orc_fermion_basis.restype = ctypes.c_long
        L.orc_fermion_basis.argtypes = [ctypes.c_int] * 3 + [_u64p, _i32p]
        L.orc_lookup_shift_from_memory.restype = ctypes.c_int
        L.orc_lookup_shift_from_memory.argtypes = [ctypes.c_int, ctypes.c_ulong]
        L.orc_fermion_lookup_table.restype = None
        L.orc_fermion_lookup_table.argtypes = [_u64p, _i32p, ctypes.c_long, ctypes.c_int, ctypes.c_int, _i32p, _i32p]
        L.orc_fermion_find_state_index.restype = ctypes.c_long
        L.orc_fermion_find_state_index.argtypes = [_u64p, ctypes.c_long, _i32p, _i32p, ctypes.c_int,
                                                   ctypes.c_uint64, ctypes.c_int]
        L.orc_fermion_aa.restype = ctypes.c_double
        L.orc_fermion_aa.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _u64p]
        L.orc_fermion_adad.restype = ctypes.c_double
        L.orc_fermion_adad.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, _u64p]
        L.orc_clebsch_gordan.restype = ctypes.c_double
        L.orc_clebsch_gordan.argtypes = [ctypes.c_int] * 5
        L.orc_nbr_pairs.restype = ctypes.c_int
        L.orc_nbr_pairs.argtypes = [ctypes.c_int]
        L.orc_interaction_tables.restype = ctypes.c_int
        L.orc_interaction_tables.argtypes = [ctypes.c_int, _f64p, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p]
        L.orc_interaction_derivatives.restype = ctypes.c_int
        L.orc_interaction_derivatives.argtypes = [ctypes.c_int, _f64p]
        L.orc_coulomb_pseudopotentials.restype = None
        L.orc_coulomb_pseudopotentials.argtypes = [ctypes.c_int, _f64p]
        L.orc_fqhe_push_add_multiply.restype = None
        L.orc_fqhe_push_add_multiply.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_long, ctypes.c_long]
        L.orc_fqhe_pull_multiply.restype = None
        L.orc_fqhe_pull_multiply.argtypes = [ctypes.c_void_p, _f64p, _f64p]
        L.orc_fqhe_row_elements.restype = ctypes.c_long
        L.orc_fqhe_row_elements.argtypes = [ctypes.c_void_p, ctypes.c_long, _i32p, _i32p, _i32p, ctypes.c_long]
        L.orc_fqhe_expectation_bins.restype = None
        L.orc_fqhe_expectation_bins.argtypes = [ctypes.c_void_p, _f64p, _f64p, _f64p]
        L.orc_spin_dimension.restype = ctypes.c_long
        L.orc_spin_dimension.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_spin_basis.restype = ctypes.c_long
        L.orc_spin_basis.argtypes = [ctypes.c_int, ctypes.c_int, _u64p]
        L.orc_spin_find_state_index.restype = ctypes.c_long
        L.orc_spin_find_state_index.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64]
        L.orc_spin_j1j2_multiply.restype = None
        L.orc_spin_j1j2_multiply.argtypes = [ctypes.c_int, ctypes.c_int, _u64p, ctypes.c_long, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, _f64p, _f64p]
        L.orc_random_vector.restype = None
        L.orc_random_vector.argtypes = [ctypes.c_uint64, ctypes.c_long, _f64p]
        L.orc_tridiagonal_eigenvalues.restype = ctypes.c_int
        L.orc_tridiagonal_eigenvalues.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p]
        L.orc_symmetric_eigen.restype = ctypes.c_int
        L.orc_symmetric_eigen.argtypes = [ctypes.c_int, _f64p, _f64p, _f64p]
        L.orc_basic_lanczos.restype = ctypes.c_int
        L.orc_basic_lanczos.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, _f64p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_double, _f64p, _i32p, _f64p, _f64p]
        L.orc_boson_unpack.restype = None
        L.orc_boson_unpack.argtypes = [ctypes.c_uint64, ctypes.c_int, _i32p]
        L.orc_boson_nbr_pairs.restype = ctypes.c_int
        L.orc_boson_nbr_pairs.argtypes = [ctypes.c_int]
        L.orc_boson_interaction_tables.restype = ctypes.c_int
        L.orc_boson_interaction_tables.argtypes = [ctypes.c_int, _f64p, _i32p, _i32p, _i32p, _i32p, _i32p, _f64p]
        L.orc_boson_push_add_multiply.restype = None
        L.orc_boson_push_add_multiply.argtypes = [ctypes.c_void_p, _f64p, _f64p, ctypes.c_long, ctypes.c_long]
        L.orc_boson_pull_multiply.restype = None
        L.orc_boson_pull_multiply.argtypes = [ctypes.c_void_p, _f64p, _f64p]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


def fermion_basis(n, two_s, total_lz):
    L = lib()
    dim = L.orc_fermion_dimension(n, total_lz, two_s)
    if dim <= 0:
        raise ValueError("empty or invalid sector N=%d 2S=%d 2Lz=%d" % (n, two_s, total_lz))
    words = np.zeros(max(dim, 1), np.uint64)
    lz = np.zeros(max(dim, 1), np.int32)
    got = L.orc_fermion_basis(n, total_lz, two_s, _p(words, _u64p), _p(lz, _i32p))
    assert got == dim
    return words[:dim], lz[:dim]


def lookup_table(words, lzmax, two_s, max_shift):
    L = lib()
    width = (1 << max_shift) + 1
    table = np.zeros((two_s + 1) * width, np.int32)
    shifts = np.zeros(two_s + 1, np.int32)
    L.orc_fermion_lookup_table(_p(words, _u64p), _p(lzmax, _i32p), len(words), two_s, max_shift,
                               _p(table, _i32p), _p(shifts, _i32p))
    return table.reshape(two_s + 1, width), shifts


def interaction_tables(two_s, v):
    L = lib()
    v = np.ascontiguousarray(v, np.float64)
    npairs = L.orc_nbr_pairs(two_s)
    cap = npairs * (two_s + 1)
    m1 = np.zeros(npairs, np.int32)
    m2 = np.zeros(npairs, np.int32)
    nm3 = np.zeros(npairs, np.int32)
    off = np.zeros(npairs, np.int32)
    m3 = np.zeros(cap, np.int32)
    fac = np.zeros(cap, np.float64)
    nf = L.orc_interaction_tables(two_s, _p(v, _f64p), _p(m1, _i32p), _p(m2, _i32p), _p(nm3, _i32p),
                                  _p(off, _i32p), _p(m3, _i32p), _p(fac, _f64p))
    return dict(m1=m1, m2=m2, nbr_m3=nm3, m3_offset=off, m3=m3[:nf], factors=fac[:nf])


def interaction_derivatives(two_s):
    L = lib()
    nf = L.orc_interaction_tables(two_s, None, None, None, None, None, None, None)
    d = np.zeros(nf * (two_s + 1), np.float64)
    L.orc_interaction_derivatives(two_s, _p(d, _f64p))
    return d.reshape(nf, two_s + 1)


def coulomb_pseudopotentials(two_s):
    v = np.zeros(two_s + 1, np.float64)
    lib().orc_coulomb_pseudopotentials(two_s, _p(v, _f64p))
    return v


def clebsch_gordan(j1, m1, j2, m2, j):
    return lib().orc_clebsch_gordan(j1, m1, j2, m2, j)


class _FqheStruct(ctypes.Structure):
    _fields_ = [("nbr_fermions", ctypes.c_int), ("lz_max", ctypes.c_int), ("total_lz", ctypes.c_int),
                ("dim", ctypes.c_long), ("words", _u64p), ("state_lz_max", _i32p), ("table", _i32p),
                ("table_shift", _i32p), ("max_shift", ctypes.c_int), ("nbr_pairs", ctypes.c_int),
                ("m1v", _i32p), ("m2v", _i32p), ("nbr_m3", _i32p), ("m3_offset", _i32p), ("m3v", _i32p),
                ("factors", _f64p), ("shift", ctypes.c_double)]


class FQHE:
    """The full FQHE sector of the oracle: basis, lookup table, interaction tables."""

    def __init__(self, n, two_s, total_lz, v, shift=0.0, max_shift=None):
        self.n, self.two_s, self.total_lz = n, two_s, total_lz
        self.words, self.lzmax = fermion_basis(n, two_s, total_lz)
        self.dim = len(self.words)
        if max_shift is None:
            max_shift = lib().orc_lookup_shift_from_memory(two_s, 9 << 20)
        self.max_shift = max_shift
        self.table, self.table_shift = lookup_table(self.words, self.lzmax, two_s, max_shift)
        self.v = np.ascontiguousarray(v, np.float64)
        self.tabs = interaction_tables(two_s, self.v)
        self.shift = shift
        t = self.tabs
        self._keep = [self.words, self.lzmax, self.table, self.table_shift, t["m1"], t["m2"], t["nbr_m3"],
                      t["m3_offset"], t["m3"], t["factors"]]
        self.s = _FqheStruct(n, two_s, total_lz, self.dim, _p(self.words, _u64p), _p(self.lzmax, _i32p),
                             _p(self.table, _i32p), _p(self.table_shift, _i32p), max_shift, len(t["m1"]),
                             _p(t["m1"], _i32p), _p(t["m2"], _i32p), _p(t["nbr_m3"], _i32p),
                             _p(t["m3_offset"], _i32p), _p(t["m3"], _i32p), _p(t["factors"], _f64p), shift)

    def find(self, word):
        w = int(word)
        lz = w.bit_length() - 1 if w else 0
        return lib().orc_fermion_find_state_index(_p(self.words, _u64p), self.dim, _p(self.table, _i32p),
                                                  _p(self.table_shift, _i32p), self.max_shift, w, lz)

    def pull(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.dim, np.float64)
        lib().orc_fqhe_pull_multiply(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p))
        return y

    def push(self, x, first=0, nbr=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.dim, np.float64)
        nbr = self.dim - first if nbr is None else nbr
        lib().orc_fqhe_push_add_multiply(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p), first, nbr)
        return y

    def row(self, r):
        cap = 4096
        t = np.zeros(cap, np.int32)
        s = np.zeros(cap, np.int32)
        f = np.zeros(cap, np.int32)
        n = lib().orc_fqhe_row_elements(ctypes.byref(self.s), r, _p(t, _i32p), _p(s, _i32p), _p(f, _i32p), cap)
        assert n <= cap
        return t[:n], s[:n], f[:n]

    def bins(self, u, v):
        u = np.ascontiguousarray(u, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        b = np.zeros(len(self.tabs["factors"]), np.float64)
        lib().orc_fqhe_expectation_bins(ctypes.byref(self.s), _p(u, _f64p), _p(v, _f64p), _p(b, _f64p))
        return b

    def lanczos(self, v0, nev=1, max_iter=200, precision=1e-14):
        return basic_lanczos(lib().orc_fqhe_matvec_cb, ctypes.byref(self.s), self.dim, v0, nev, max_iter, precision)


def boson_interaction_tables(two_s, v):
    """The bosonic factors of ParticleOnSphereGenericHamiltonian (:620-806), layout of interaction_tables
    with pairs m1 >= m2."""
    L = lib()
    v = np.ascontiguousarray(v, np.float64)
    npairs = L.orc_boson_nbr_pairs(two_s)
    cap = npairs * (two_s + 1)
    m1 = np.zeros(npairs, np.int32)
    m2 = np.zeros(npairs, np.int32)
    nm3 = np.zeros(npairs, np.int32)
    off = np.zeros(npairs, np.int32)
    m3 = np.zeros(cap, np.int32)
    fac = np.zeros(cap, np.float64)
    nf = L.orc_boson_interaction_tables(two_s, _p(v, _f64p), _p(m1, _i32p), _p(m2, _i32p), _p(nm3, _i32p),
                                        _p(off, _i32p), _p(m3, _i32p), _p(fac, _f64p))
    return dict(m1=m1, m2=m2, nbr_m3=nm3, m3_offset=off, m3=m3[:nf], factors=fac[:nf])


def boson_occupations(words, two_s):
    out = np.zeros((len(words), two_s + 1), np.int32)
    for i, w in enumerate(words):
        lib().orc_boson_unpack(int(w), two_s, _p(out[i], _i32p))
    return out


class BosonFQHE(FQHE):
    """N bosons in 2S + 1 orbitals at 2Lz, BosonOnSphereShort representation: the words and lookup
    table of FermionOnSphere(N, 2Lz, 2S + N - 1) and the bosonic interaction tables."""

    def __init__(self, n, two_s, total_lz, v, shift=0.0):
        self.n, self.two_s, self.total_lz = n, two_s, total_lz
        lzf = two_s + n - 1
        self.words, self.lzmax = fermion_basis(n, lzf, total_lz)
        self.dim = len(self.words)
        self.max_shift = lib().orc_lookup_shift_from_memory(lzf, 9 << 20)
        self.table, self.table_shift = lookup_table(self.words, self.lzmax, lzf, self.max_shift)
        self.v = np.ascontiguousarray(v, np.float64)
        self.tabs = boson_interaction_tables(two_s, self.v)
        self.shift = shift
        t = self.tabs
        self._keep = [self.words, self.lzmax, self.table, self.table_shift, t["m1"], t["m2"], t["nbr_m3"],
                      t["m3_offset"], t["m3"], t["factors"]]
        self.s = _FqheStruct(n, lzf, total_lz, self.dim, _p(self.words, _u64p), _p(self.lzmax, _i32p),
                             _p(self.table, _i32p), _p(self.table_shift, _i32p), self.max_shift, len(t["m1"]),
                             _p(t["m1"], _i32p), _p(t["m2"], _i32p), _p(t["nbr_m3"], _i32p),
                             _p(t["m3_offset"], _i32p), _p(t["m3"], _i32p), _p(t["factors"], _f64p), shift)

    def occupations(self):
        return boson_occupations(self.words, self.two_s)

    def pull(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.dim, np.float64)
        lib().orc_boson_pull_multiply(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p))
        return y

    def push(self, x, first=0, nbr=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.dim, np.float64)
        nbr = self.dim - first if nbr is None else nbr
        lib().orc_boson_push_add_multiply(ctypes.byref(self.s), _p(x, _f64p), _p(y, _f64p), first, nbr)
        return y

    def lanczos(self, v0, nev=1, max_iter=200, precision=1e-14):
        return basic_lanczos(lib().orc_boson_matvec_cb, ctypes.byref(self.s), self.dim, v0, nev, max_iter, precision)


def spin_basis(length, sz):
    L = lib()
    dim = L.orc_spin_dimension(length, sz)
    w = np.zeros(dim, np.uint64)
    L.orc_spin_basis(length, sz, _p(w, _u64p))
    return w


def spin_find(length, sz, word):
    return lib().orc_spin_find_state_index(length, sz, int(word))


def spin_j1j2_multiply(length, sz, words, j1, j2, x, shift=0.0):
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(len(words), np.float64)
    lib().orc_spin_j1j2_multiply(length, sz, _p(words, _u64p), len(words), j1, j2, shift, _p(x, _f64p), _p(y, _f64p))
    return y


def random_vector(seed, dim):
    x = np.zeros(dim, np.float64)
    lib().orc_random_vector(seed, dim, _p(x, _f64p))
    return x


def tridiagonal_eigenvalues(diag, off):
    d = np.ascontiguousarray(diag, np.float64)
    e = np.ascontiguousarray(off, np.float64)
    out = np.zeros(len(d), np.float64)
    assert lib().orc_tridiagonal_eigenvalues(len(d), _p(d, _f64p), _p(e, _f64p), _p(out, _f64p)) == 0
    return out


_MATVEC_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, _f64p, _f64p)


def basic_lanczos(fn, ctx, dim, v0, nev=1, max_iter=200, precision=1e-14):
    v0 = np.ascontiguousarray(v0, np.float64)
    eig = np.zeros(nev, np.float64)
    it = np.zeros(1, np.int32)
    alpha = np.zeros(max_iter + 8, np.float64)
    beta = np.zeros(max_iter + 8, np.float64)
    conv = lib().orc_basic_lanczos(ctypes.cast(fn, ctypes.c_void_p), ctx, dim, _p(v0, _f64p), nev, max_iter,
                                   precision, _p(eig, _f64p), _p(it, _i32p), _p(alpha, _f64p), _p(beta, _f64p))
    return dict(eigenvalues=eig, iterations=int(it[0]), converged=bool(conv))


def python_lanczos(matvec, dim, v0, nev=1, max_iter=200, precision=1e-14):
    """Basic Lanczos with a Python matvec callable (for the spin chain)."""
    @_MATVEC_CB
    def cb(ctx, x, y):
        xa = np.ctypeslib.as_array(x, shape=(dim,))
        ya = np.ctypeslib.as_array(y, shape=(dim,))
        ya[:] = matvec(xa)
    r = basic_lanczos(cb, None, dim, v0, nev, max_iter, precision)
    return r


def l2_factors(n, two_s, total_lz):
    """L^2 = L-L+ + Lz^2 + Lz of N fermions in 2S+1 orbitals as a two-body table in the layout of
    interaction_tables (pairs m1 > m2, creation m3 > M/2, element = F(m1, m2, m3) <t|a+_m3 a+_m4
    a_m1 a_m2|s>, the operator the reference's ParticleOnSphereL2Hamiltonian applies,
    ParticleOnSphereL2Hamiltonian.cc:240-368): L+ = sum_m lam_m a+_{m+1} a_m, so
    L-L+ = sum_m lam_m^2 n_m - sum_{m,m'} lam_m lam_m' a+_m' a+_{m+1} a_{m'+1} a_m, each term put in
    canonical order with its fermionic sign; the one-body part is folded into the diagonal pair
    factors (sum_m w_m n_m = sum_{a>b} (w_a + w_b) / (N - 1) n_a n_b at fixed N).  Returns
    (factors, constant) with constant = Lz^2 + Lz, Lz = total_lz / 2."""
    t = interaction_tables(two_s, np.zeros(two_s + 1))
    lam = [0.5 * np.sqrt(two_s * (two_s + 2) - (2 * m - two_s) * (2 * m - two_s + 2)) for m in range(two_s + 1)]
    F = {}

    def add(c, d, a, val):
        F[(c, d, a)] = F.get((c, d, a), 0.0) + val

    for m in range(two_s):
        for mp in range(two_s):
            if mp == m + 1 or mp + 1 == m:
                continue
            a_, b_, s1 = (mp, m + 1, 1.0) if mp > m + 1 else (m + 1, mp, -1.0)
            c_, d_, s2 = (mp + 1, m, 1.0) if mp + 1 > m else (m, mp + 1, -1.0)
            add(c_, d_, a_, -lam[m] * lam[mp] * s1 * s2)
    w = [lam[m] ** 2 for m in range(two_s + 1)]
    for a_ in range(two_s + 1):
        for b_ in range(a_):
            add(a_, b_, a_, -(w[a_] + w[b_]) / (n - 1))
    f = np.zeros_like(t["factors"])
    for p in range(len(t["m1"])):
        m1, m2 = int(t["m1"][p]), int(t["m2"][p])
        for q in range(int(t["nbr_m3"][p])):
            f[t["m3_offset"][p] + q] = F.get((m1, m2, int(t["m3"][t["m3_offset"][p] + q])), 0.0)
    lz = total_lz / 2.0
    return f, lz * lz + lz


def boson_l2_factors(n, two_s, total_lz):
    """L^2 of N bosons as a two-body table in the layout of boson_interaction_tables (pairs m1 >= m2,
    creation m3 >= M/2, element = F(m1, m2, m3) <t|a+_m3 a+_m4 a_m1 a_m2|s>), the reference's bosonic
    branch of ParticleOnSphereL2Hamiltonian (ParticleOnSphereL2Hamiltonian.cc:240-368).  Bosons
    commute, so L-L+ = sum_m lam_m^2 n_m + sum_{m,m'} lam_m lam_m' a+_m' a+_{m+1} a_{m'+1} a_m with no
    sign; at fixed N the one-body part is sum_{a>b} (w_a + w_b) / (N - 1) n_a n_b +
    sum_a w_a / (N - 1) n_a (n_a - 1).  Returns (factors, Lz^2 + Lz)."""
    t = boson_interaction_tables(two_s, np.zeros(two_s + 1))
    lam = [0.5 * np.sqrt(two_s * (two_s + 2) - (2 * m - two_s) * (2 * m - two_s + 2)) for m in range(two_s + 1)]
    F = {}

    def add(c, d, a, val):
        F[(c, d, a)] = F.get((c, d, a), 0.0) + val

    for m in range(two_s):
        for mp in range(two_s):
            add(max(mp + 1, m), min(mp + 1, m), max(mp, m + 1), lam[m] * lam[mp])
    w = [lam[m] ** 2 for m in range(two_s + 1)]
    for a_ in range(two_s + 1):
        for b_ in range(a_):
            add(a_, b_, a_, (w[a_] + w[b_]) / (n - 1))
        add(a_, a_, a_, w[a_] / (n - 1))
    f = np.zeros_like(t["factors"])
    slots = set()
    for p in range(len(t["m1"])):
        m1, m2 = int(t["m1"][p]), int(t["m2"][p])
        for q in range(int(t["nbr_m3"][p])):
            key = (m1, m2, int(t["m3"][t["m3_offset"][p] + q]))
            slots.add(key)
            f[t["m3_offset"][p] + q] = F.get(key, 0.0)
    assert all(k in slots for k in F), "an L^2 term outside the bosonic table"
    lz = total_lz / 2.0
    return f, lz * lz + lz


def l2_raise(n, two_s, total_lz, x):
    """L+ x from the sector 2Lz to 2Lz + 2: a+_{m+1} a_m hops with coefficient lam_m and sign +1
    (no orbital lies between m and m + 1)."""
    words, _ = fermion_basis(n, two_s, total_lz)
    up, _ = fermion_basis(n, two_s, total_lz + 2)
    index = {int(w): i for i, w in enumerate(up)}
    y = np.zeros(len(up))
    for i, w in enumerate(words):
        w = int(w)
        for m in range(two_s):
            if (w >> m) & 1 and not (w >> (m + 1)) & 1:
                lam = 0.5 * np.sqrt(two_s * (two_s + 2) - (2 * m - two_s) * (2 * m - two_s + 2))
                y[index[w ^ (3 << m)]] += lam * x[i]
    return y


def read_vector_bytes(b):
    """A vector file's bytes (RealVector::WriteVector, src/Vector/RealVector.cc:3669): int32
    dimension, or int32 -1 and an int64 dimension, then little-endian doubles."""
    d = int(np.frombuffer(b[:4], "<i4")[0])
    off = 4
    if d <= 0 and len(b) > 4:
        d = int(np.frombuffer(b[4:12], "<i8")[0])
        off = 12
    assert len(b) == off + 8 * d, (len(b), d)
    return np.frombuffer(b[off:], "<f8").copy()


def read_lanczos_state(b, fmt):
    """lanczos.dat bytes of the reference's disk-storage Lanczos classes.
    fmt "basic": BasicLanczosAlgorithmWithDiskStorage::WriteState (BasicLanczosAlgorithmWithDiskStorage.cc:
    286-308): int32 Index, f64 PreviousLastWantedEigenvalue, f64 EigenvaluePrecision, int32 NbrRow, three
    NUL-terminated vector file names, Index+2 diagonal then Index+1 upper-diagonal elements.
    fmt "ground": BasicLanczosAlgorithmWithGroundStateDiskStorage::WriteState (...GroundStateDiskStorage.cc:
    399-423): int32 Index, int32 GroundStateEvaluationFlag, f64 PreviousLastWantedEigenvalue, f64
    EigenvaluePrecision, int32 NbrEigenvalue, int32 NbrRow, NbrRow diagonal then NbrRow-1 upper-diagonal
    elements."""
    b = bytes(b)
    if fmt == "basic":
        index = int(np.frombuffer(b[0:4], "<i4")[0])
        prev, prec = np.frombuffer(b[4:20], "<f8")
        nbr_row = int(np.frombuffer(b[20:24], "<i4")[0])
        names, o = [], 24
        for _ in range(3):
            e = b.index(b"\0", o)
            names.append(b[o:e].decode())
            o = e + 1
        rows = index + 2
        diag = np.frombuffer(b[o:o + 8 * rows], "<f8").copy()
        upper = np.frombuffer(b[o + 8 * rows:o + 8 * (2 * rows - 1)], "<f8").copy()
        assert len(b) == o + 8 * (2 * rows - 1)
        return dict(index=index, prev_last=float(prev), precision=float(prec), nbr_row=nbr_row, names=names,
                    diag=diag, upper=upper, ground_flag=0)
    index, flag = (int(x) for x in np.frombuffer(b[0:8], "<i4"))
    prev, prec = np.frombuffer(b[8:24], "<f8")
    nev, nbr_row = (int(x) for x in np.frombuffer(b[24:32], "<i4"))
    diag = np.frombuffer(b[32:32 + 8 * nbr_row], "<f8").copy()
    upper = np.frombuffer(b[32 + 8 * nbr_row:], "<f8").copy()
    assert upper.size == nbr_row - 1
    return dict(index=index, ground_flag=flag, prev_last=float(prev), precision=float(prec), nbr_eigenvalue=nev,
                nbr_row=nbr_row, diag=diag, upper=upper)


def entanglement_matrix(n, two_s, total_lz, x, l, na, lza):
    """The orbital-cut entanglement matrix of FermionOnSphere::EvaluatePartialEntanglementMatrix
    (FermionOnSphere.cc:2474) restated with the oracle's bases: A = orbitals 0..l-1 in the sector
    (na, lza), rows in FermionOnSphere(na, lza, l - 1) order, columns in the complement's order, M[a][b]
    = x of the state a | (b << l).  Regular cuts only (0 < l <= 2S)."""
    words, _ = fermion_basis(n, two_s, total_lz)
    nb = n - na
    sum_a = (lza + na * (l - 1)) // 2  # floored, as the reference does (FermionOnSphere.cc:2095)
    lza = 2 * sum_a - na * (l - 1)
    sum_b = (total_lz + n * two_s) // 2 - sum_a
    if na > l or nb > two_s + 1 - l or not (na * (na - 1) // 2 <= sum_a <= na * (l - 1) - na * (na - 1) // 2):
        return np.zeros((0, 0))
    if not (l * nb + nb * (nb - 1) // 2 <= sum_b <= nb * two_s - nb * (nb - 1) // 2):
        return np.zeros((0, 0))
    a_words = fermion_basis(na, l - 1, lza)[0] if na > 0 else np.zeros(1, np.uint64)
    lz_b = 2 * (sum_b - nb * l) - nb * (two_s - l)
    b_words = fermion_basis(nb, two_s - l, lz_b)[0] if nb > 0 else np.zeros(1, np.uint64)
    ra = {int(w): i for i, w in enumerate(a_words)}
    rb = {int(w): i for i, w in enumerate(b_words)}
    m = np.zeros((len(a_words), len(b_words)))
    mask = (1 << l) - 1
    for i, w in enumerate(words):
        w = int(w)
        a, b = w & mask, w >> l
        if a in ra and b in rb:
            m[ra[a], rb[b]] = x[i]
    return m


def _translation_canonical(w, L):
    """Spin1_2ChainWithTranslations::FindCanonicalForm (.h:478) and FindNumberTranslation (:530): the
    first smallest of the L rotations of w (one site each), the rotations to it, and the orbit size."""
    c, n, orbit, t = w, 0, L, w
    for k in range(1, L):
        t = (t >> 1) | ((t & 1) << (L - 1))
        if t == w and orbit == L:
            orbit = k
        if t < c:
            c, n = t, k
    return c, n, orbit


def translation_basis(L, sz, k):
    """Spin1_2ChainWithTranslations(L, k, 1, sz) (Spin1_2ChainWithTranslations.cc:167-235): the words
    with (L + sz) / 2 up spins that are their own canonical form and whose orbit size o satisfies
    k o = 0 mod L, ascending; returns (words, orbit sizes)."""
    from itertools import combinations
    n_up = (L + sz) // 2
    words = sorted(sum(1 << p for p in c) for c in combinations(range(L), n_up))
    reps, orbits = [], []
    for w in words:
        c, _, o = _translation_canonical(w, L)
        if c == w and (o * k) % L == 0:
            reps.append(w)
            orbits.append(o)
    return np.array(reps, np.uint64), np.array(orbits, np.int32)


def translation_j1j2_push(L, sz, k, j1, j2, x):
    """SpinChainJ1J2RealHamiltonianWithTranslations::LowLevelAddMultiply (.cc:94-192) restated: for every
    representative s and every bond (J1: i, i+1; J2: i, i+2, periodic) with antiparallel spins, the flipped
    word's representative t receives J/2 sqrt(o_s / o_t) cos(2 pi k ((L - n) mod L) / L) x[s] (SymmetrizeResult,
    Spin1_2ChainWithTranslations.h:419); plus the SzSz diagonal (:335-352)."""
    reps, orbits = translation_basis(L, sz, k)
    index = {int(w): i for i, w in enumerate(reps)}
    y = np.zeros(len(reps))
    phase = [np.cos(2.0 * np.pi / L * k * m) for m in range(L)]
    for i, w in enumerate(reps):
        w = int(w)
        diag = 0.0
        for dist, j in ((1, j1), (2, j2)):
            for a in range(L):
                b = (a + dist) % L
                if ((w >> a) & 1) == ((w >> b) & 1):
                    diag += 0.25 * j
                    continue
                diag -= 0.25 * j
                f = w ^ ((1 << a) | (1 << b))
                c, n, o = _translation_canonical(f, L)
                t = index.get(c)
                if t is None:
                    continue
                y[t] += 0.5 * j * np.sqrt(orbits[i] / orbits[t]) * phase[(L - n) % L] * x[i]
        y[i] += diag * x[i]
    return y


def translation_flip_count(L, sz, k):
    """Number of spin flips of the J1-J2 chain (both bond types) from a representative whose word lies in
    the momentum sector: the off-diagonal elements SymmetrizeResult keeps
    (SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192)."""
    reps, _ = translation_basis(L, sz, k)
    index = set(int(w) for w in reps)
    kept = 0
    for w in reps:
        w = int(w)
        for dist in (1, 2):
            for a in range(L):
                b = (a + dist) % L
                if ((w >> a) & 1) != ((w >> b) & 1):
                    kept += _translation_canonical(w ^ ((1 << a) | (1 << b)), L)[0] in index
    return kept


# ------------------------------------------------------------------ FermionOnSphereLong (128-bit words)
# Python integers stand for ULONGLONG words; small sectors only.

def fermion_basis_long(n, two_s, total_lz):
    """FermionOnSphereLong::GenerateStates (FermionOnSphereLong.cc:911-943) restated: every word of n
    fermions in orbitals 0..two_s with orbital sum (total_lz + n two_s) / 2, highest fermion placed as
    high as possible first (descending words)."""
    total = total_lz + n * two_s
    if total < 0 or total & 1:
        raise ValueError("sector not reachable")
    out = []

    def rec(k, top, s, prefix):
        if k == 0:
            if s == 0:
                out.append(prefix)
            return
        for q in range(top, k - 2, -1):
            rest = s - q
            if rest < (k - 1) * (k - 2) // 2:
                continue
            if rest > (k - 1) * (q - 1) - (k - 1) * (k - 2) // 2:
                break
            rec(k - 1, q - 1, rest, prefix | (1 << q))

    rec(n, two_s, total // 2, 0)
    return out


def _parity(x):
    return -1.0 if bin(x).count("1") & 1 else 1.0


def fermion_aa_long(state, n1, n2):
    """FermionOnSphereLong::AA (FermionOnSphereLong.cc:553): annihilate n2 then n1, each sign the parity
    of the occupied orbitals at and above the annihilated one; (coefficient, word)."""
    if n1 == n2 or not (state >> n1) & 1 or not (state >> n2) & 1:
        return 0.0, 0
    c = _parity(state >> n2)
    state &= ~(1 << n2)
    c *= _parity(state >> n1)
    return c, state & ~(1 << n1)


def fermion_adad_long(state, m1, m2):
    """FermionOnSphereLong::AdAd (FermionOnSphereLong.cc:647): create m2 then m1, each sign the parity
    of the occupied orbitals above the created one; (coefficient, word)."""
    if (state >> m2) & 1:
        return 0.0, 0
    c = _parity(state >> m2)
    state |= 1 << m2
    if (state >> m1) & 1:
        return 0.0, 0
    c *= _parity(state >> m1)
    return c, state | (1 << m1)


class FQHELong:
    """ParticleOnSphereGenericHamiltonian on FermionOnSphereLong, push form of
    AbstractQHEOnSphereHamiltonian::LowLevelAddMultiply (AbstractQHEOnSphereHamiltonian.cc:456-488), with
    the interaction tables of interaction_tables(); FindStateIndex by a dictionary."""

    def __init__(self, n, two_s, total_lz, v, shift=0.0):
        self.words = fermion_basis_long(n, two_s, total_lz)
        self.index = {w: i for i, w in enumerate(self.words)}
        self.dim = len(self.words)
        self.shift = shift
        t = interaction_tables(two_s, v)
        self.moves = []
        for p in range(len(t["m1"])):
            m1, m2 = int(t["m1"][p]), int(t["m2"][p])
            o, k = int(t["m3_offset"][p]), int(t["nbr_m3"][p])
            self.moves.append((m1, m2, [(int(t["m3"][o + q]), float(t["factors"][o + q])) for q in range(k)]))

    def push(self, x, first=0, nbr=None):
        nbr = self.dim - first if nbr is None else nbr
        y = np.zeros(self.dim)
        for i in range(first, first + nbr):
            s = self.words[i]
            for m1, m2, creations in self.moves:
                c, a = fermion_aa_long(s, m1, m2)
                if c == 0.0:
                    continue
                c *= x[i]
                for m3, f in creations:
                    c2, t = fermion_adad_long(a, m3, m1 + m2 - m3)
                    if c2 != 0.0:
                        y[self.index[t]] += c * f * c2
            y[i] += self.shift * x[i]
        return y


def translation_j1j2_push_complex(L, sz, k, j1, j2, x):
    """SpinChainJ1J2HamiltonianWithTranslations::LowLevelAddMultiply (.cc:149-247) restated for any
    momentum k: for every representative s and antiparallel bond, the flipped word's representative t
    receives J/2 sqrt(o_s / o_t) exp(2 pi i k m / L) x[s], m = (L - n) mod L the translation count that
    SymmetrizeResult returns (Spin1_2ChainWithTranslations.h:421-432); plus the SzSz diagonal.  x and the
    result are complex."""
    reps, orbits = translation_basis(L, sz, k)
    index = {int(w): i for i, w in enumerate(reps)}
    x = np.asarray(x, np.complex128)
    y = np.zeros(len(reps), np.complex128)
    phase = [np.exp(2j * np.pi / L * k * m) for m in range(L)]
    for i, w in enumerate(reps):
        w = int(w)
        diag = 0.0
        for dist, j in ((1, j1), (2, j2)):
            for a in range(L):
                b = (a + dist) % L
                if ((w >> a) & 1) == ((w >> b) & 1):
                    diag += 0.25 * j
                    continue
                diag -= 0.25 * j
                c, n, o = _translation_canonical(w ^ ((1 << a) | (1 << b)), L)
                t = index.get(c)
                if t is None:
                    continue
                y[t] += 0.5 * j * np.sqrt(orbits[i] / orbits[t]) * phase[(L - n) % L] * x[i]
        y[i] += diag * x[i]
    return y
