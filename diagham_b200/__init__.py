"""diagham_b200: DiagHam's on-the-fly H.v + Lanczos path on one B200.

Python view of the C ABI in include/diagham_b200.h (libdiagham_b200.so, built in this directory by
diagham_b200/_build.py).  Class and method names follow the reference classes they replace:

    FermionOnSphere                     FQHE/src/HilbertSpace/FermionOnSphere.h
    FermionOnSphereLong                 FQHE/src/HilbertSpace/FermionOnSphereLong.h
    BosonOnSphereShort                  FQHE/src/HilbertSpace/BosonOnSphereShort.h
    Spin1_2Chain                        Spin/src/HilbertSpace/Spin1_2Chain.h
    ParticleOnSphereGenericHamiltonian  FQHE/src/Hamiltonian/ParticleOnSphereGenericHamiltonian.h
    SpinChainJ1J2Hamiltonian            (J1-J2 pattern of SpinChainJ1J2RealHamiltonianWithTranslations on a plain chain)
    Spin1_2ChainWithTranslations, SpinChainJ1J2RealHamiltonianWithTranslations,
    SpinChainJ1J2HamiltonianWithTranslations
                                        Spin/src/HilbertSpace, Spin/src/Hamiltonian (momentum sectors)
    BasicLanczosAlgorithm, FullReorthogonalizedLanczosAlgorithm, BasicLanczosAlgorithmWithGroundState,
    BasicLanczosAlgorithmWithDiskStorage, BasicLanczosAlgorithmWithGroundStateDiskStorage
                                        src/LanczosAlgorithm/*.h
    WriteVector, ReadVector             RealVector::WriteVector / ReadVector (src/Vector/RealVector.cc)

Vectors are FP64 numpy arrays (host) or torch CUDA tensors (used in place).  Every call goes to
the GPU; there is no CPU fallback: importing without the built library raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdiagham_b200.so")

DH_OK = 0
# launch forms of the split-word FQHE kernel (dh_hamiltonian_autotune's last result)
SPLIT_FORMS = ["256x4", "256x3", "256x3 pipelined", "256x2 pipelined", "128x8", "256x2", "192x4", "128x6"]
DH_INDEX_RANK = 0
DH_INDEX_LOOKUP = 1
DH_PRECISION_FP64 = 0
DH_PRECISION_FP32 = 1
DH_LANCZOS_BASIC = 0
DH_LANCZOS_FULL_REORTHOGONALIZED = 1
DH_LANCZOS_BLOCK = 2
DH_LANCZOS_WITH_GROUND_STATE = 3

# every exported entry point with its argument types (restype int unless stated)
_c_int, _c_dbl, _c_i64, _c_u64, _vp = ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)
SIGNATURES = {
    "dh_last_error": ([], ctypes.c_char_p),
    "dh_version": ([], ctypes.c_char_p),
    "dh_device_count": ([_ip], _c_int),
    "dh_fermion_on_sphere_create": ([_c_int, _c_int, _c_int, ctypes.c_ulong, _vp], _c_int),
    "dh_boson_on_sphere_create": ([_c_int, _c_int, _c_int, ctypes.c_ulong, _vp], _c_int),
    "dh_spin12_chain_create": ([_c_int, _c_int, _c_int, _vp], _c_int),
    "dh_spin12_chain_translations_create": ([_c_int, _c_int, _c_int, _c_int, _vp], _c_int),
    "dh_space_destroy": ([_vp], _c_int),
    "dh_space_get_dimension": ([_vp, _i64p], _c_int),
    "dh_space_get_states": ([_vp, _vp, _vp, _c_i64, _c_i64], _c_int),
    "dh_space_find_state_index": ([_vp, _vp, _c_i64, _vp], _c_int),
    "dh_fermion_on_sphere_long_create": ([_c_int, _c_int, _c_int, ctypes.c_ulong, _vp], _c_int),
    "dh_space_get_states_long": ([_vp, _vp, _vp, _c_i64, _c_i64], _c_int),
    "dh_complex_vector_write": ([ctypes.c_char_p, _vp, _c_i64], _c_int),
    "dh_complex_vector_file_dimension": ([ctypes.c_char_p, _vp], _c_int),
    "dh_complex_vector_read": ([ctypes.c_char_p, _vp, _c_i64], _c_int),
    "dh_space_find_state_index_long": ([_vp, _vp, _c_i64, _vp], _c_int),
    "dh_space_set_index_mode": ([_vp, _c_int], _c_int),
    "dh_space_set_split_form": ([_vp, _c_int], _c_int),
    "dh_fermion_on_sphere_partial_entanglement_matrix": ([_vp, _vp, _c_int, _c_int, _c_int, _vp, _c_i64, _i64p, _i64p],
                                                         _c_int),
    "dh_fermion_on_sphere_partial_density_matrix": ([_vp, _vp, _c_int, _c_int, _c_int, _vp, _c_i64, _i64p], _c_int),
    "dh_particle_on_sphere_generic_hamiltonian_create": ([_vp, _c_int, _c_int, _vp, _c_dbl, _vp], _c_int),
    "dh_particle_on_sphere_l2_hamiltonian_create": ([_vp, _c_int, _c_int, _c_int, _c_dbl, _vp], _c_int),
    "dh_spin_chain_j1j2_hamiltonian_create": ([_vp, _c_dbl, _c_dbl, _vp], _c_int),
    "dh_spin_chain_j1j2_complex_hamiltonian_create": ([_vp, _c_dbl, _c_dbl, _vp], _c_int),
    "dh_hamiltonian_destroy": ([_vp], _c_int),
    "dh_hamiltonian_get_dimension": ([_vp, _i64p], _c_int),
    "dh_hamiltonian_shift": ([_vp, _c_dbl], _c_int),
    "dh_hamiltonian_set_precision": ([_vp, _c_int], _c_int),
    "dh_hamiltonian_set_pseudopotentials": ([_vp, _vp], _c_int),
    "dh_hamiltonian_set_stream": ([_vp, _vp], _c_int),
    "dh_hamiltonian_low_level_add_multiply": ([_vp, _vp, _vp, _c_i64, _c_i64], _c_int),
    "dh_hamiltonian_low_level_multiply": ([_vp, _vp, _vp, _c_i64, _c_i64], _c_int),
    "dh_hamiltonian_low_level_multiple_add_multiply": ([_vp, _vp, _vp, _c_int, _c_i64, _c_i64], _c_int),
    "dh_hamiltonian_block_multiply": ([_vp, _vp, _vp, _c_int], _c_int),
    "dh_hamiltonian_autotune": ([_vp, _c_int, _c_int, _vp], _c_int),
    "dh_hamiltonian_enable_fast_multiplication": ([_vp, _c_i64, _ip, _i64p], _c_int),
    "dh_hamiltonian_disable_fast_multiplication": ([_vp], _c_int),
    "dh_hamiltonian_matrix_element": ([_vp, _vp, _vp, _vp], _c_int),
    "dh_hamiltonian_row_elements": ([_vp, _c_i64, _vp, _vp, _vp, _c_int, _ip], _c_int),
    "dh_hamiltonian_pseudopotential_adjoint": ([_vp, _vp, _vp, _vp], _c_int),
    "dh_hamiltonian_get_interaction_factors": ([_vp, _vp, _c_int, _ip], _c_int),
    "dh_hamiltonian_pseudopotential_adjoint_static": ([_vp, _vp, _vp, _vp], _c_int),
    "dh_hamiltonian_count_elements": ([_vp, _i64p], _c_int),
    "dh_hamiltonian_count_diagonal_elements": ([_vp, _i64p], _c_int),
    "dh_lanczos_create": ([_vp, _c_int, _c_int, _c_int, _c_int, _vp], _c_int),
    "dh_lanczos_destroy": ([_vp], _c_int),
    "dh_lanczos_set_eigenvalue_precision": ([_vp, _c_dbl], _c_int),
    "dh_lanczos_set_vector_storage": ([_vp, _c_int], _c_int),
    "dh_lanczos_initialize": ([_vp, _vp, _c_int], _c_int),
    "dh_lanczos_initialize_random": ([_vp, _c_u64], _c_int),
    "dh_lanczos_run": ([_vp, _c_int], _c_int),
    "dh_lanczos_test_convergence": ([_vp, _ip], _c_int),
    "dh_lanczos_get_eigenvalues": ([_vp, _vp, _c_int], _c_int),
    "dh_lanczos_get_ground_state_energy": ([_vp, _vp], _c_int),
    "dh_lanczos_get_ground_state": ([_vp, _vp], _c_int),
    "dh_lanczos_get_eigenstates": ([_vp, _c_int, _vp], _c_int),
    "dh_lanczos_get_counters": ([_vp, _i64p, _ip], _c_int),
    "dh_lanczos_solve": ([_vp, _c_int, _c_int, _vp, _ip, _ip], _c_int),
    "dh_lanczos_solve_refined": ([_vp, _c_int, _c_dbl, _vp], _c_int),
    "dh_hamiltonian_tune_block_size": ([_vp, _c_int, _c_dbl, _c_int, _vp, _vp], _c_int),
    "dh_lanczos_set_disk_storage": ([_vp, ctypes.c_char_p, _c_int], _c_int),
    "dh_lanczos_write_state": ([_vp], _c_int),
    "dh_lanczos_resume": ([_vp], _c_int),
    "dh_vector_write": ([ctypes.c_char_p, _vp, _c_i64], _c_int),
    "dh_vector_file_dimension": ([ctypes.c_char_p, _i64p], _c_int),
    "dh_vector_read": ([ctypes.c_char_p, _vp, _c_i64], _c_int),
    "dh_fqhe_sectors_block_lanczos": ([_c_int, _c_int, _vp, _c_int, _vp, _c_int, _c_int, _c_dbl, _c_int, _c_int,
                                       _c_i64, _c_u64, _vp, _vp, _vp], _c_int),
    "dh_coulomb_pseudopotentials": ([_c_int, _vp], _c_int),
    "dh_clebsch_gordan": ([_c_int, _c_int, _c_int, _c_int, _c_int, _vp], _c_int),
}

_lib = None


class DiagHamError(RuntimeError):
    pass


def library_path():
    return _LIB_PATH


def load(path=None):
    """Load libdiagham_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or _LIB_PATH
    if not os.path.exists(p):
        raise DiagHamError("libdiagham_b200.so is not built: run python -m diagham_b200._build (or __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _check(rc):
    if rc != DH_OK:
        msg = _lib.dh_last_error().decode(errors="replace")
        raise DiagHamError("error %d: %s" % (rc, msg))


def version():
    return load().dh_version().decode()


def device_count():
    n = ctypes.c_int(0)
    _check(load().dh_device_count(ctypes.byref(n)))
    return n.value


class _Buf:
    """A pointer to FP64 (or other) data: numpy (host) or torch CUDA tensor (device, in place)."""

    def __init__(self, a, dtype=np.float64, writable=False, size=None):
        self.keep = None
        self.out = None
        if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
            import torch
            want = {np.float64: torch.float64, np.uint64: torch.int64, np.int64: torch.int64}[dtype]
            if a.is_cuda:
                if a.dtype != want or not a.is_contiguous():
                    raise TypeError("CUDA tensors must be contiguous %s" % want)
                self.ptr = a.data_ptr()
                self.n = a.numel()
                return
            a = a.detach().numpy()
        arr = np.ascontiguousarray(a, dtype=dtype)
        if writable and arr is not a:
            self.out = a
        self.keep = arr
        self.ptr = arr.ctypes.data
        self.n = arr.size

    def finish(self):
        if self.out is not None:
            self.out[...] = self.keep.reshape(self.out.shape)


class _Space:
    _handle = None

    def GetHilbertSpaceDimension(self):
        d = ctypes.c_int64(0)
        _check(_lib.dh_space_get_dimension(self._handle, ctypes.byref(d)))
        return d.value

    @property
    def dim(self):
        return self.GetHilbertSpaceDimension()

    def states(self, first=0, n=None):
        """(StateDescription, StateLzMax) of states first..first+n, reference layout."""
        d = self.dim
        n = d - first if n is None else n
        words = np.zeros(n, np.uint64)
        lz = np.zeros(n, np.int32)
        _check(_lib.dh_space_get_states(self._handle, words.ctypes.data, lz.ctypes.data, first, n))
        return words, lz

    def FindStateIndex(self, words):
        w = _Buf(words, np.uint64)
        out = np.zeros(w.n, np.int64)
        _check(_lib.dh_space_find_state_index(self._handle, w.ptr, w.n, out.ctypes.data))
        return out

    def set_index_mode(self, mode):
        m = {"rank": DH_INDEX_RANK, "lookup": DH_INDEX_LOOKUP}.get(mode, mode)
        _check(_lib.dh_space_set_index_mode(self._handle, m))

    def set_split_form(self, form):
        """Launch form of the split-word product kernel (an index into SPLIT_FORMS or its name)."""
        f = SPLIT_FORMS.index(form) if isinstance(form, str) else int(form)
        _check(_lib.dh_space_set_split_form(self._handle, f))

    def __del__(self):
        if self._handle and _lib is not None:
            _lib.dh_space_destroy(self._handle)
            self._handle = None


class FermionOnSphere(_Space):
    """FermionOnSphere(nbrFermions, totalLz, lzMax, memory): FermionOnSphere.cc:75."""

    def __init__(self, nbr_fermions, total_lz, lz_max, memory=9 << 20):
        load()
        h = ctypes.c_void_p()
        _check(_lib.dh_fermion_on_sphere_create(nbr_fermions, total_lz, lz_max, memory, ctypes.byref(h)))
        self._handle = h
        self.nbr_fermions, self.total_lz, self.lz_max = nbr_fermions, total_lz, lz_max

    def EvaluatePartialEntanglementMatrix(self, subsystem_size, nbr_fermion_sector, lz_sector, state):
        """M[a][b] of the orbital cut at subsystem_size (FermionOnSphere.cc:2474), (rows, cols)."""
        return _cut_matrix(self, _lib.dh_fermion_on_sphere_partial_entanglement_matrix, state,
                           (subsystem_size, nbr_fermion_sector, lz_sector), False)

    def EvaluatePartialDensityMatrix(self, subsystem_size, nbr_fermion_sector, lz_sector, state):
        """rho_A = M M^T of the orbital cut (FermionOnSphere.cc:2070)."""
        return _cut_matrix(self, _lib.dh_fermion_on_sphere_partial_density_matrix, state,
                           (subsystem_size, nbr_fermion_sector, lz_sector), True)


class FermionOnSphereLong(_Space):
    """FermionOnSphereLong(nbrFermions, totalLz, lzMax, memory): FermionOnSphereLong.cc:67, lzMax up to
    126.  states() gives the 128-bit words as an (n, 2) uint64 array of (low, high) halves;
    FindStateIndex takes such pairs or Python integers (-1 outside the sector)."""

    def __init__(self, nbr_fermions, total_lz, lz_max, memory=9 << 20):
        load()
        h = ctypes.c_void_p()
        _check(_lib.dh_fermion_on_sphere_long_create(nbr_fermions, total_lz, lz_max, memory, ctypes.byref(h)))
        self._handle = h
        self.nbr_fermions, self.total_lz, self.lz_max = nbr_fermions, total_lz, lz_max

    def states(self, first=0, n=None):
        d = self.dim
        n = d - first if n is None else n
        words = np.zeros((n, 2), np.uint64)
        lz = np.zeros(n, np.int32)
        _check(_lib.dh_space_get_states_long(self._handle, words.ctypes.data, lz.ctypes.data, first, n))
        return words, lz

    @staticmethod
    def word_values(pairs):
        """Python integers of (low, high) pairs."""
        return [int(a) | (int(b) << 64) for a, b in np.asarray(pairs, np.uint64).reshape(-1, 2)]

    @staticmethod
    def word_pairs(values):
        """(n, 2) uint64 (low, high) pairs of Python integers."""
        m = (1 << 64) - 1
        return np.array([[v & m, v >> 64] for v in values], np.uint64).reshape(-1, 2)

    def FindStateIndex(self, words):
        if not (isinstance(words, np.ndarray) and words.dtype == np.uint64 and words.ndim == 2):
            words = self.word_pairs([int(w) for w in words])
        words = np.ascontiguousarray(words, np.uint64)
        out = np.zeros(words.shape[0], np.int64)
        _check(_lib.dh_space_find_state_index_long(self._handle, words.ctypes.data, words.shape[0], out.ctypes.data))
        return out


def _cut_matrix(space, fn, state, args, square):
    b = _Buf(state)
    r, c = ctypes.c_int64(0), ctypes.c_int64(0)
    sizes = (ctypes.byref(r),) if square else (ctypes.byref(r), ctypes.byref(c))
    _check(fn(space._handle, b.ptr, *args, None, 0, *sizes))
    rows, cols = r.value, (r.value if square else c.value)
    out = np.zeros((rows, cols), np.float64)
    if out.size:
        _check(fn(space._handle, b.ptr, *args, out.ctypes.data, out.size, *sizes))
    return out


class BosonOnSphereShort(_Space):
    """BosonOnSphereShort(nbrBosons, totalLz, lzMax): BosonOnSphereShort.cc:81.  states() and
    FindStateIndex use the FermionOnSphere words of the occupations (n_0 ones, a zero, n_1 ones, ...)."""

    def __init__(self, nbr_bosons, total_lz, lz_max, memory=0):
        load()
        h = ctypes.c_void_p()
        _check(_lib.dh_boson_on_sphere_create(nbr_bosons, total_lz, lz_max, memory, ctypes.byref(h)))
        self._handle = h
        self.nbr_bosons, self.total_lz, self.lz_max = nbr_bosons, total_lz, lz_max

    def occupations(self, words):
        """Occupations n_0..n_lzmax of each word (rows of an (n, lz_max + 1) array)."""
        words = np.asarray(words, np.uint64)
        out = np.zeros((words.size, self.lz_max + 1), np.int32)
        for i, w in enumerate(words):
            w, m = int(w), 0
            while m <= self.lz_max:
                c = 0
                while w & 1:
                    c += 1
                    w >>= 1
                out[i, m] = c
                w >>= 1
                m += 1
        return out


class Spin1_2Chain(_Space):
    """Spin1_2Chain(chainLength, sz, memorySize): Spin1_2Chain.cc:113."""

    def __init__(self, chain_length, sz, memory=1 << 20):
        load()
        h = ctypes.c_void_p()
        _check(_lib.dh_spin12_chain_create(chain_length, sz, memory, ctypes.byref(h)))
        self._handle = h
        self.chain_length, self.sz = chain_length, sz


class _Hamiltonian:
    _handle = None

    def GetHilbertSpaceDimension(self):
        d = ctypes.c_int64(0)
        _check(_lib.dh_hamiltonian_get_dimension(self._handle, ctypes.byref(d)))
        return d.value

    @property
    def dim(self):
        return self.GetHilbertSpaceDimension()

    def ShiftHamiltonian(self, shift):
        _check(_lib.dh_hamiltonian_shift(self._handle, float(shift)))

    def set_precision(self, precision):
        p = {"fp64": DH_PRECISION_FP64, "fp32": DH_PRECISION_FP32}.get(precision, precision)
        _check(_lib.dh_hamiltonian_set_precision(self._handle, p))

    def set_stream(self, stream):
        _check(_lib.dh_hamiltonian_set_stream(self._handle, ctypes.c_void_p(stream)))

    def LowLevelAddMultiply(self, src, dst, first=0, nbr=-1):
        s, d = _Buf(src), _Buf(dst, writable=True)
        _check(_lib.dh_hamiltonian_low_level_add_multiply(self._handle, s.ptr, d.ptr, first, nbr))
        d.finish()
        return dst

    def LowLevelMultiply(self, src, dst=None, first=0, nbr=-1):
        if dst is None:
            dst = np.zeros(self.dim, np.float64)
        s, d = _Buf(src), _Buf(dst, writable=True)
        _check(_lib.dh_hamiltonian_low_level_multiply(self._handle, s.ptr, d.ptr, first, nbr))
        d.finish()
        return dst

    def LowLevelMultipleAddMultiply(self, srcs, dsts, first=0, nbr=-1):
        """srcs, dsts: (k, dim) arrays (k vectors one after the other)."""
        k = srcs.shape[0]
        s, d = _Buf(srcs), _Buf(dsts, writable=True)
        _check(_lib.dh_hamiltonian_low_level_multiple_add_multiply(self._handle, s.ptr, d.ptr, k, first, nbr))
        d.finish()
        return dsts

    def block_multiply(self, x, y=None):
        """y = H x for a row-interleaved block x of shape (dim, k) (numpy or torch CUDA)."""
        k = 1 if len(x.shape) == 1 else int(x.shape[1])
        if y is None:
            y = np.zeros((self.dim, k), np.float64) if isinstance(x, np.ndarray) else x.new_empty(x.shape)
        s, d = _Buf(x), _Buf(y, writable=True)
        _check(_lib.dh_hamiltonian_block_multiply(self._handle, s.ptr, d.ptr, k))
        d.finish()
        return y

    def EnableFastMultiplication(self, allowed_memory=-1):
        """Store every row's elements in device memory if they fit in allowed_memory bytes (< 0: no
        budget).  Returns (enabled, bytes needed)."""
        en = ctypes.c_int(0)
        nb = ctypes.c_int64(0)
        _check(_lib.dh_hamiltonian_enable_fast_multiplication(self._handle, int(allowed_memory), ctypes.byref(en),
                                                              ctypes.byref(nb)))
        return bool(en.value), nb.value

    def DisableFastMultiplication(self):
        _check(_lib.dh_hamiltonian_disable_fast_multiplication(self._handle))

    def autotune(self, block_size=1, repeats=3):
        """Time the product's kernel forms on this Hamiltonian and keep the fastest one."""
        out = np.zeros(11, np.float64)
        _check(_lib.dh_hamiltonian_autotune(self._handle, block_size, repeats, out.ctypes.data))
        return dict(best_ms=out[0], kernel_variant={0: "split", 1: "generic", 2: "split+smem"}[int(out[1])],
                    low_bits=int(out[2]), ms_k1=out[3], ms_k2=out[4], ms_k4=out[5], candidates=int(out[6]),
                    stored_ms=out[7], stored_in_use=bool(out[8]), launch_form=SPLIT_FORMS[int(out[9])],
                    stored_read_ahead=int(out[10]))

    def tune_block_size(self, max_iter=600, precision=1e-10, refined=True):
        """Block size (1, 2 or 4) with the shortest time to the converged ground energy, and the times."""
        k = ctypes.c_int(0)
        t = np.zeros(3, np.float64)
        _check(_lib.dh_hamiltonian_tune_block_size(self._handle, int(max_iter), float(precision), int(bool(refined)),
                                                   ctypes.byref(k), t.ctypes.data))
        return k.value, dict(zip((1, 2, 4), t.tolist()))

    def count_elements(self):
        """Elements one product generates (moves incl. diagonal ones; spin flips)."""
        t = ctypes.c_int64(0)
        _check(_lib.dh_hamiltonian_count_elements(self._handle, ctypes.byref(t)))
        return t.value

    def count_diagonal_elements(self):
        """Of count_elements(), those that return to their own row."""
        t = ctypes.c_int64(0)
        _check(_lib.dh_hamiltonian_count_diagonal_elements(self._handle, ctypes.byref(t)))
        return t.value

    def MatrixElement(self, v1, v2):
        a, b = _Buf(v1), _Buf(v2)
        out = ctypes.c_double(0.0)
        _check(_lib.dh_hamiltonian_matrix_element(self._handle, a.ptr, b.ptr, ctypes.byref(out)))
        return out.value

    def __del__(self):
        if self._handle and _lib is not None:
            _lib.dh_hamiltonian_destroy(self._handle)
            self._handle = None


class ParticleOnSphereGenericHamiltonian(_Hamiltonian):
    """ParticleOnSphereGenericHamiltonian(particles, nbrParticles, lzmax, pseudoPotential, l2Factor):
    ParticleOnSphereGenericHamiltonian.cc:66 with on-the-fly multiplication."""

    def __init__(self, space, nbr_particles, lz_max, pseudopotentials, l2_factor=0.0):
        load()
        self.space = space  # the Hamiltonian does not own the space; keep it alive
        v = np.ascontiguousarray(pseudopotentials, np.float64)
        if v.size != lz_max + 1:
            raise ValueError("need lz_max + 1 pseudopotentials")
        h = ctypes.c_void_p()
        _check(_lib.dh_particle_on_sphere_generic_hamiltonian_create(space._handle, nbr_particles, lz_max,
                                                                     v.ctypes.data, float(l2_factor), ctypes.byref(h)))
        self._handle = h
        self.lz_max = lz_max

    def set_pseudopotentials(self, v):
        v = np.ascontiguousarray(v, np.float64)
        _check(_lib.dh_hamiltonian_set_pseudopotentials(self._handle, v.ctypes.data))

    def row_elements(self, row, cap=8192):
        t = np.zeros(cap, np.int32)
        s = np.zeros(cap, np.int32)
        f = np.zeros(cap, np.int32)
        n = ctypes.c_int(0)
        _check(_lib.dh_hamiltonian_row_elements(self._handle, row, t.ctypes.data, s.ctypes.data, f.ctypes.data, cap,
                                                ctypes.byref(n)))
        if n.value > cap:
            return self.row_elements(row, n.value)
        return t[:n.value], s[:n.value], f[:n.value]

    def interaction_factors(self):
        n = ctypes.c_int(0)
        _check(_lib.dh_hamiltonian_get_interaction_factors(self._handle, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value, np.float64)
        _check(_lib.dh_hamiltonian_get_interaction_factors(self._handle, out.ctypes.data, n.value, ctypes.byref(n)))
        return out

    def pseudopotential_adjoint(self, u, v):
        """out[m] = <u| dH/dV_m |v>."""
        a, b = _Buf(u), _Buf(v)
        out = np.zeros(self.lz_max + 1, np.float64)
        _check(_lib.dh_hamiltonian_pseudopotential_adjoint(self._handle, a.ptr, b.ptr, out.ctypes.data))
        return out


    def pseudopotential_adjoint_static(self, u, v):
        """pseudopotential_adjoint without any device allocation (u, v must be CUDA tensors); its
        scratch is a static device array shared by all calls, so concurrent calls race."""
        a, b = _Buf(u), _Buf(v)
        out = np.zeros(self.lz_max + 1, np.float64)
        _check(_lib.dh_hamiltonian_pseudopotential_adjoint_static(self._handle, a.ptr, b.ptr, out.ctypes.data))
        return out


class ParticleOnSphereL2Hamiltonian(_Hamiltonian):
    """ParticleOnSphereL2Hamiltonian(particles, nbrParticles, lzmax, totalLz, l2Factor) with Lz fixed
    by the sector: l2_factor L^2 (ParticleOnSphereL2Hamiltonian.cc:240-368)."""

    def __init__(self, space, nbr_particles, lz_max, total_lz, l2_factor=1.0):
        load()
        self.space = space
        self.lz_max = lz_max
        h = ctypes.c_void_p()
        _check(_lib.dh_particle_on_sphere_l2_hamiltonian_create(space._handle, nbr_particles, lz_max, total_lz,
                                                                float(l2_factor), ctypes.byref(h)))
        self._handle = h
        self.l2_factor = l2_factor

    def total_angular_momentum(self, psi):
        """L with <psi|L^2|psi> / <psi|psi> = L (L + 1)."""
        psi = np.asarray(psi.detach().cpu() if hasattr(psi, "detach") else psi, np.float64)
        l2 = self.MatrixElement(psi, psi) / float(psi @ psi) / self.l2_factor
        return 0.5 * (np.sqrt(1.0 + 4.0 * max(l2, 0.0)) - 1.0)


class Spin1_2ChainWithTranslations(_Space):
    """Spin1_2ChainWithTranslations(chainLength, momentum, 1, sz, memory, memorySlice): the momentum
    sector of the periodic chain (Spin1_2ChainWithTranslations.cc:167); states() gives the
    representatives (smallest word of each orbit), ascending."""

    def __init__(self, chain_length, momentum, sz, memory=1 << 20):
        load()
        h = ctypes.c_void_p()
        _check(_lib.dh_spin12_chain_translations_create(chain_length, momentum, sz, memory, ctypes.byref(h)))
        self._handle = h
        self.chain_length, self.momentum, self.sz = chain_length, momentum, sz


class SpinChainJ1J2Hamiltonian(_Hamiltonian):
    """Periodic J1-J2 chain on a plain Spin1_2Chain (element pattern of
    SpinChainJ1J2RealHamiltonianWithTranslations.cc:94-192, API of SpinChainHamiltonian.cc:257)."""

    def __init__(self, chain, j1, j2):
        load()
        self.space = chain
        h = ctypes.c_void_p()
        _check(_lib.dh_spin_chain_j1j2_hamiltonian_create(chain._handle, float(j1), float(j2), ctypes.byref(h)))
        self._handle = h


class _Lanczos:
    ALGORITHM = DH_LANCZOS_BASIC
    _handle = None

    def __init__(self, hamiltonian, nbr_eigenvalue=1, max_iter=500, block_size=1):
        load()
        self.hamiltonian = hamiltonian
        self.nbr_eigenvalue = nbr_eigenvalue
        h = ctypes.c_void_p()
        _check(_lib.dh_lanczos_create(hamiltonian._handle, self.ALGORITHM, nbr_eigenvalue, block_size, max_iter,
                                      ctypes.byref(h)))
        self._handle = h

    def set_vector_storage(self, keep):
        _check(_lib.dh_lanczos_set_vector_storage(self._handle, 1 if keep else 0))

    def SetEigenvaluePrecision(self, precision):
        _check(_lib.dh_lanczos_set_eigenvalue_precision(self._handle, float(precision)))

    def InitializeLanczosAlgorithm(self, vector=None, seed=0):
        """No vector: a reproducible random start from seed.  A vector (dim,) or vectors
        (nbr, dim) (numpy or torch CUDA): the start vector(s); block algorithms complete and
        orthonormalise the block."""
        if vector is None:
            _check(_lib.dh_lanczos_initialize_random(self._handle, seed))
        else:
            b = _Buf(vector)
            nbr = 1 if len(vector.shape) == 1 else int(vector.shape[0])
            _check(_lib.dh_lanczos_initialize(self._handle, b.ptr, nbr))

    def RunLanczosAlgorithm(self, nbr_iter):
        _check(_lib.dh_lanczos_run(self._handle, nbr_iter))

    def TestConvergence(self):
        c = ctypes.c_int(0)
        _check(_lib.dh_lanczos_test_convergence(self._handle, ctypes.byref(c)))
        return bool(c.value)

    def GetEigenvalues(self, n=None):
        n = self.nbr_eigenvalue if n is None else n
        out = np.zeros(n, np.float64)
        _check(_lib.dh_lanczos_get_eigenvalues(self._handle, out.ctypes.data, n))
        return out

    def GetGroundStateEnergy(self):
        e = ctypes.c_double(0.0)
        _check(_lib.dh_lanczos_get_ground_state_energy(self._handle, ctypes.byref(e)))
        return e.value

    def GetGroundState(self, out=None):
        dim = self.hamiltonian.dim
        if out is None:
            out = np.zeros(dim, np.float64)
        b = _Buf(out, writable=True)
        _check(_lib.dh_lanczos_get_ground_state(self._handle, b.ptr))
        b.finish()
        return out

    def GetEigenstates(self, n, out=None):
        """The n lowest Ritz vectors, normalised, as an (n, dim) array (or into out)."""
        dim = self.hamiltonian.dim
        if out is None:
            out = np.zeros((n, dim), np.float64)
        b = _Buf(out, writable=True)
        _check(_lib.dh_lanczos_get_eigenstates(self._handle, n, b.ptr))
        b.finish()
        return out

    def counters(self):
        m = ctypes.c_int64(0)
        r = ctypes.c_int(0)
        _check(_lib.dh_lanczos_get_counters(self._handle, ctypes.byref(m), ctypes.byref(r)))
        return m.value, r.value

    def solve(self, max_iter=500, graph_batch=16):
        """Driver loop of QHEOnSphereMainTask.cc:732-753 on the device."""
        eig = np.zeros(self.nbr_eigenvalue, np.float64)
        it = ctypes.c_int(0)
        conv = ctypes.c_int(0)
        _check(_lib.dh_lanczos_solve(self._handle, max_iter, graph_batch, eig.ctypes.data, ctypes.byref(it),
                                     ctypes.byref(conv)))
        return dict(eigenvalues=eig, iterations=it.value, converged=bool(conv.value))

    def solve_refined(self, max_iter=500, precision=1e-12):
        """FP32-product Lanczos, then FP64 refinement of the ground state."""
        out = np.zeros(5, np.float64)
        _check(_lib.dh_lanczos_solve_refined(self._handle, max_iter, float(precision), out.ctypes.data))
        return dict(energy=out[0], energy_fp32=out[1], residual=out[2], fp32_matvecs=int(out[3]),
                    fp64_matvecs=int(out[4]))

    def set_disk_storage(self, directory, interval=1):
        """Checkpoint the state into `directory` in the reference's disk-storage format of this
        algorithm, every `interval` rows and at the end of solve; None switches it off."""
        d = None if directory is None else os.fsencode(directory)
        _check(_lib.dh_lanczos_set_disk_storage(self._handle, d, int(interval)))

    def WriteState(self):
        _check(_lib.dh_lanczos_write_state(self._handle))

    def ResumeLanczosAlgorithm(self):
        _check(_lib.dh_lanczos_resume(self._handle))

    def __del__(self):
        if self._handle and _lib is not None:
            _lib.dh_lanczos_destroy(self._handle)
            self._handle = None


class BasicLanczosAlgorithmWithDiskStorage(_Lanczos):
    """BasicLanczosAlgorithmWithDiskStorage(architecture, nbrEigenvalue, maxIter): the basic algorithm
    with its state in `directory` (lanczos.dat and three vector files) after every `interval` rows."""
    ALGORITHM = DH_LANCZOS_BASIC

    def __init__(self, hamiltonian, nbr_eigenvalue=1, max_iter=500, directory=".", interval=1):
        super().__init__(hamiltonian, nbr_eigenvalue, max_iter)
        self.set_disk_storage(directory, interval)


class BasicLanczosAlgorithmWithGroundStateDiskStorage(_Lanczos):
    """BasicLanczosAlgorithmWithGroundStateDiskStorage(architecture, nbrIter, maxIter): the ground-state
    algorithm with its state in `directory` (lanczos.dat, vector.0 = start vector, vector.1-3)."""
    ALGORITHM = DH_LANCZOS_WITH_GROUND_STATE

    def __init__(self, hamiltonian, max_iter=500, directory=".", interval=1):
        super().__init__(hamiltonian, 1, max_iter)
        self.set_disk_storage(directory, interval)


class BasicLanczosAlgorithm(_Lanczos):
    ALGORITHM = DH_LANCZOS_BASIC


class FullReorthogonalizedLanczosAlgorithm(_Lanczos):
    ALGORITHM = DH_LANCZOS_FULL_REORTHOGONALIZED


class BasicLanczosAlgorithmWithGroundState(_Lanczos):
    ALGORITHM = DH_LANCZOS_WITH_GROUND_STATE


class BasicBlockLanczosAlgorithm(_Lanczos):
    """BasicBlockLanczosAlgorithm(architecture, nbrEigenvalue, blockSize, maxIter): block_size 1, 2
    or 4 vectors per step, one product per block step for the whole block."""
    ALGORITHM = DH_LANCZOS_BLOCK

    def __init__(self, hamiltonian, nbr_eigenvalue=1, max_iter=500, block_size=2):
        super().__init__(hamiltonian, nbr_eigenvalue, max_iter, block_size)
        self.block_size = block_size


def coulomb_pseudopotentials(nbr_flux):
    """EvaluatePseudopotentials(nbrFlux, 0, 0.0): LLL Coulomb V_0..V_nbrFlux on the sphere."""
    load()
    v = np.zeros(nbr_flux + 1, np.float64)
    _check(_lib.dh_coulomb_pseudopotentials(nbr_flux, v.ctypes.data))
    return v


def clebsch_gordan(j1, m1, j2, m2, j):
    load()
    out = ctypes.c_double(0.0)
    _check(_lib.dh_clebsch_gordan(j1, m1, j2, m2, j, ctypes.byref(out)))
    return out.value


def fqhe_sectors_block_lanczos(nbr_fermions, lz_max, total_lz, pseudopotentials, block_size=4, max_iter=400,
                               precision=1e-14, fp32=False, full_diag_limit=200, seed=100, memory=0):
    """Lowest energy of every requested Lz sector: block Lanczos over all sectors in lockstep, one
    launch per block product (BasicBlockLanczosAlgorithm + QHEOnSphereMainTask's loop per sector).
    fp32=True: FP32 products, then FP64 refinement of every sector to `precision`.  memory: bytes the
    stored elements of the whole batch may take (the reference's --memory; 0: on the fly, < 0: as
    much as fits)."""
    load()
    tl = np.ascontiguousarray(total_lz, np.int32)
    v = np.ascontiguousarray(pseudopotentials, np.float64)
    ns = tl.size
    e = np.zeros(ns, np.float64)
    it = np.zeros(ns, np.int32)
    secs = np.zeros(12, np.float64)
    _check(_lib.dh_fqhe_sectors_block_lanczos(nbr_fermions, lz_max, tl.ctypes.data, ns, v.ctypes.data, block_size,
                                              max_iter, float(precision),
                                              DH_PRECISION_FP32 if fp32 else DH_PRECISION_FP64, full_diag_limit,
                                              int(memory), seed, e.ctypes.data, it.ctypes.data, secs.ctypes.data))
    return dict(energies=e, iterations=it, setup_seconds=secs[0], solve_seconds=secs[1], product_seconds=secs[2],
                block_products=int(secs[3]), fp32_seconds=secs[4], refine_seconds=secs[5],
                refined_sectors=int(secs[6]), max_refine_shift=secs[7], dense_fallback_sectors=int(secs[8]),
                dense_fallback_seconds=secs[9], stored_bytes=int(secs[10]), store_seconds=secs[11])


def WriteVector(vec, file_name):
    """RealVector::WriteVector: vec (numpy or torch CUDA, FP64) into file_name; a complex numpy vector is
    written as ComplexVector::WriteVector writes it."""
    load()
    if isinstance(vec, np.ndarray) and np.iscomplexobj(vec):
        pairs = np.ascontiguousarray(vec, np.complex128).view(np.float64)
        _check(_lib.dh_complex_vector_write(os.fsencode(file_name), pairs.ctypes.data, vec.size))
        return
    b = _Buf(vec)
    _check(_lib.dh_vector_write(os.fsencode(file_name), b.ptr, b.n))


def vector_file_dimension(file_name):
    load()
    d = ctypes.c_int64(0)
    _check(_lib.dh_vector_file_dimension(os.fsencode(file_name), ctypes.byref(d)))
    return d.value


def ReadComplexVector(file_name):
    """ComplexVector::ReadVector: the complex vector stored in file_name (numpy complex128)."""
    load()
    d = ctypes.c_int64(0)
    _check(_lib.dh_complex_vector_file_dimension(os.fsencode(file_name), ctypes.byref(d)))
    out = np.zeros(d.value, np.complex128)
    _check(_lib.dh_complex_vector_read(os.fsencode(file_name), out.view(np.float64).ctypes.data, d.value))
    return out


def ReadVector(file_name, out=None):
    """RealVector::ReadVector: the vector stored in file_name (into out if given: numpy or torch
    CUDA of the stored dimension)."""
    dim = vector_file_dimension(file_name)
    if out is None:
        out = np.zeros(dim, np.float64)
    b = _Buf(out, writable=True)
    _check(_lib.dh_vector_read(os.fsencode(file_name), b.ptr, b.n))
    b.finish()
    return out


def eigenstate_file_name(statistics, interaction_name, nbr_particles, lz_max, total_lz, index):
    """<statistics>_<interaction>_n_<N>_2s_<2S>_lz_<2Lz>.<index>.vec, the eigenstate naming of
    FQHE/docs/DataFormat/FermionOnSphere.xml:9-16 (statistics "fermions" or "bosons", total_lz = 2 Lz)."""
    return "%s_%s_n_%d_2s_%d_lz_%d.%d.vec" % (statistics, interaction_name, nbr_particles, lz_max, total_lz, index)


def spectrum_file_name(statistics, interaction_name, nbr_particles, lz_max, extra_terms=""):
    """<statistics>_<interaction><extra>_n_<N>_2s_<2S>_lz.dat, the spectrum file of the sphere programs
    (FQHESphereFermionsTwoBodyGeneric.cc:243)."""
    return "%s_%s%s_n_%d_2s_%d_lz.dat" % (statistics, interaction_name, extra_terms, nbr_particles, lz_max)


def back_up_file(file_name, extension=".bak"):
    """BackUpFile (src/GeneralTools/FilenameTools.cc:381): an existing file_name is renamed to
    file_name.bak, or file_name.bak1, .bak2, ... (the first free name); returns the counter, -1 when
    there was nothing to back up."""
    if not os.path.exists(file_name):
        return -1
    counter, target = 0, file_name + extension
    while os.path.exists(target):
        counter += 1
        target = "%s%s%d" % (file_name, extension, counter)
    os.rename(file_name, target)
    return counter


def _stream_double(x):
    # a double through a C++ stream in its default format at precision 14
    return "%.14g" % x


class QHEOnSphereSpectrumFile:
    """The spectrum file QHEOnSphereMainTask::ExecuteMainTask writes (QHEOnSphereMainTask.cc:361-456): the
    first sector backs up an existing file and writes the header "# Lz E" (with " <H>" when the energies are
    also evaluated on the eigenvectors, " <L^2> <L>" with the total angular momentum), then every
    eigenvalue of a sector is a line "LValue/2 E" (LValue = 2 Lz, integer division as in C++; E minus
    the energy shift; doubles at 14 significant digits), followed by <H> and <L^2> L when given."""

    def __init__(self, file_name, energy_column=False, l_value_columns=False):
        self.file_name = file_name
        back_up_file(file_name)
        header = "# Lz E" + (" <H>" if energy_column else "") + (" <L^2> <L>" if l_value_columns else "")
        with open(file_name, "w") as f:
            f.write(header + "\n")

    def add(self, two_lz, energies, energy_shift=0.0, expectations=None, l2_values=None):
        lz = int(two_lz / 2)  # truncation toward zero, as LValue / 2 on ints
        with open(self.file_name, "a") as f:
            for j, e in enumerate(energies):
                line = "%d %s" % (lz, _stream_double(e - energy_shift))
                if expectations is not None:
                    line += " " + _stream_double(expectations[j] - energy_shift)
                if l2_values is not None:
                    l2 = float(l2_values[j])
                    line += " %s %s" % (_stream_double(l2), _stream_double(0.5 * (np.sqrt(4.0 * l2 + 1.0) - 1.0)))
                f.write(line + "\n")


class SpinChainJ1J2HamiltonianWithTranslations(_Hamiltonian):
    """SpinChainJ1J2HamiltonianWithTranslations(chain, nbrSpin, j1, j2)
    (SpinChainJ1J2HamiltonianWithTranslations.cc:62): the complex Hamiltonian of a momentum sector, any
    K.  Products take and return complex vectors (numpy complex128; float64 arrays or torch CUDA
    tensors of 2 D (Re, Im) pairs are taken as they are), with first / nbr counting complex
    components.  dim is 2 D: the Lanczos classes run on the (Re, Im) form and give ground states in it
    (as_complex turns them into complex arrays)."""

    def __init__(self, chain, nbr_spin, j1, j2):
        load()
        if nbr_spin != chain.chain_length:
            raise ValueError("nbr_spin must be the chain length")
        self.space = chain
        h = ctypes.c_void_p()
        _check(_lib.dh_spin_chain_j1j2_complex_hamiltonian_create(chain._handle, float(j1), float(j2),
                                                                  ctypes.byref(h)))
        self._handle = h

    @staticmethod
    def as_complex(v):
        v = v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v)
        return np.ascontiguousarray(v, np.float64).view(np.complex128)

    @staticmethod
    def _real(v):
        if isinstance(v, np.ndarray) and np.iscomplexobj(v):
            return np.ascontiguousarray(v, np.complex128).view(np.float64)
        return v

    def LowLevelAddMultiply(self, src, dst, first=0, nbr=-1):
        out = self._real(dst)
        super().LowLevelAddMultiply(self._real(src), out, 2 * first, 2 * nbr if nbr >= 0 else -1)
        return dst

    def LowLevelMultiply(self, src, dst=None, first=0, nbr=-1):
        if dst is None:
            dst = np.zeros(self.dim // 2, np.complex128)
        super().LowLevelMultiply(self._real(src), self._real(dst), 2 * first, 2 * nbr if nbr >= 0 else -1)
        return dst

    def LowLevelMultipleAddMultiply(self, srcs, dsts, first=0, nbr=-1):
        s, d = self._real(srcs), self._real(dsts)
        super().LowLevelMultipleAddMultiply(s, d, 2 * first, 2 * nbr if nbr >= 0 else -1)
        return dsts

    def MatrixElement(self, v1, v2):
        """Re <v1|H|v2>."""
        return super().MatrixElement(self._real(v1), self._real(v2))


class SpinChainJ1J2RealHamiltonianWithTranslations(SpinChainJ1J2Hamiltonian):
    """SpinChainJ1J2RealHamiltonianWithTranslations(chain, nbrSpin, j1, j2)
    (SpinChainJ1J2RealHamiltonianWithTranslations.cc:58) on a Spin1_2ChainWithTranslations space,
    momentum 0 or L / 2."""

    def __init__(self, chain, nbr_spin, j1, j2):
        if nbr_spin != chain.chain_length:
            raise ValueError("nbr_spin must be the chain length")
        super().__init__(chain, j1, j2)
