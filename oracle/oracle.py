"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product (dmg-md_b200/) never does.

  OracleModel   -- FP64 restatement in oracle/nep_oracle.c
  RefCpuModel   -- the reference's own NEP3_CPU evaluator (FP64), compiled
                   from its sources into oracle/_ref/ by oracle/Makefile
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libnep_oracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libnep_ref_cpu.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build():
    """Compile the oracle (and, when the reference tree is present, oracle/_ref)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load(ORACLE_SO)
        _lib.nepo_load.restype = ctypes.c_void_p
        _lib.nepo_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        _lib.nepo_free.argtypes = [ctypes.c_void_p]
        _lib.nepo_info.argtypes = [ctypes.c_void_p, _i32p, _f64p]
        _lib.nepo_compute.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _f64p, _i32p, _f64p,
                                      _f64p, _f64p, _f64p]
        _lib.nepo_descriptors.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _f64p, _i32p,
                                          _f64p, _f64p]
        _lib.nepo_neighbors_f32.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _f64p, _i32p,
                                            _f64p, ctypes.c_int, ctypes.c_int, _i32p, _i32p]
        _lib.nepo_harmonic_tables.argtypes = [_f64p, _f64p]
    return _lib


def harmonic_tables():
    """(z[9, 9, 9], c3b[80]): z-polynomial coefficients [L][m][power] and q_L weights."""
    z = np.zeros((9, 9, 9))
    c3b = np.zeros(80)
    lib().nepo_harmonic_tables(z, c3b)
    return z, c3b


def _prep(types, h, pbc, pos):
    types = np.ascontiguousarray(types, dtype=np.int32)
    h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(9))
    pbc = np.ascontiguousarray(pbc if pbc is not None else [1, 1, 1], dtype=np.int32)
    pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float64).reshape(3, -1))
    return types, h, pbc, pos


class OracleModel:
    """FP64 NEP evaluation of one structure (positions SoA, shape (3, n))."""

    def __init__(self, path):
        err = ctypes.create_string_buffer(512)
        self._h = lib().nepo_load(os.fsencode(path), err, 512)
        if not self._h:
            raise ValueError(err.value.decode())
        info = np.zeros(16, dtype=np.int32)
        rc = np.zeros(32, dtype=np.float64)
        lib().nepo_info(self._h, info, rc)
        keys = ["version", "num_types", "zbl", "zbl_flexible", "n_max_r", "n_max_a", "basis_r",
                "basis_a", "L_max", "num_L", "dim", "H", "MN_r", "MN_a", "has_q", "typewise_zbl"]
        self.info = dict(zip(keys, (int(v) for v in info)))
        t = self.info["num_types"]
        self.rc_radial = rc[0:2 * t:2].copy()
        self.rc_angular = rc[1:2 * t:2].copy()

    def __del__(self):
        if getattr(self, "_h", None):
            lib().nepo_free(self._h)
            self._h = None

    def compute(self, types, h, pos, pbc=None):
        types, h, pbc, pos = _prep(types, h, pbc, pos)
        n = types.size
        pe = np.zeros(n)
        force = np.zeros(3 * n)
        virial = np.zeros(9 * n)
        rc = lib().nepo_compute(self._h, n, types, h, pbc, pos.reshape(-1), pe, force, virial)
        if rc:
            raise RuntimeError("oracle compute failed")
        return pe, force.reshape(3, n), virial.reshape(9, n)

    def descriptors(self, types, h, pos, pbc=None):
        types, h, pbc, pos = _prep(types, h, pbc, pos)
        n = types.size
        q = np.zeros(n * self.info["dim"])
        lib().nepo_descriptors(self._h, n, types, h, pbc, pos.reshape(-1), q)
        return q.reshape(n, self.info["dim"])

    def neighbors_f32(self, types, h, pos, which, mn=None, pbc=None):
        """Sorted typewise neighbour rows (list of int arrays), FP32 predicate."""
        types, h, pbc, pos = _prep(types, h, pbc, pos)
        n = types.size
        mn = mn or (self.info["MN_r"] if which == 0 else self.info["MN_a"])
        nn = np.zeros(n, dtype=np.int32)
        nl = np.zeros(n * mn, dtype=np.int32)
        if lib().nepo_neighbors_f32(self._h, n, types, h, pbc, pos.reshape(-1), which, mn, nn, nl):
            raise RuntimeError("neighbour row overflow")
        nl = nl.reshape(n, mn)
        return [nl[i, :nn[i]].copy() for i in range(n)]


_ref = None


def ref_cpu_available():
    return os.path.exists(REF_CPU_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_CPU_SO)
        _ref.nepref_create.restype = ctypes.c_void_p
        _ref.nepref_create.argtypes = [ctypes.c_char_p]
        _ref.nepref_destroy.argtypes = [ctypes.c_void_p]
    return _ref


class RefCpuModel:
    """The reference's NEP3_CPU (FP64), driven through oracle/ref_cpu_driver.cpp.

    compute(..., threads=T, center_begin/end) evaluates the centers
    [begin, end) with T host threads; forces and virials are folded back from
    periodic ghosts onto their owners.
    """

    def __init__(self, path):
        self._h = ref_lib().nepref_create(os.fsencode(path))
        if not self._h:
            raise ValueError("NEP3_CPU could not load %s" % path)

    def __del__(self):
        if getattr(self, "_h", None):
            ref_lib().nepref_destroy(self._h)
            self._h = None

    def compute(self, types, h, pos, threads=1, center_begin=0, center_end=None):
        types, h, _, pos = _prep(types, h, None, pos)
        n = types.size
        end = n if center_end is None else center_end
        pe = np.zeros(n)
        force = np.zeros(3 * n)
        virial = np.zeros(9 * n)
        rc = self._compute(n, types, h, pos, threads, center_begin, end, pe, force, virial)
        if rc:
            raise RuntimeError("NEP3_CPU compute failed (%d)" % rc)
        return pe, force.reshape(3, n), virial.reshape(9, n)

    def _compute(self, n, types, h, pos, threads, begin, end, pe, force, virial):
        f = ref_lib().nepref_compute_range
        f.restype = ctypes.c_int
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, _i32p, _f64p, _f64p, ctypes.c_int,
                      ctypes.c_int, ctypes.c_int, _f64p, _f64p, _f64p]
        return f(self._h, n, types, h, pos.reshape(-1), threads, begin, end, pe, force, virial)


REF_GPU_SO = os.path.join(HERE, "_ref", "libnep_ref_gpu.so")
_refgpu = None


def ref_gpu_available():
    return os.path.exists(REF_GPU_SO)


def refgpu_lib():
    global _refgpu
    if _refgpu is None:
        L = ctypes.CDLL(REF_GPU_SO)
        vp = ctypes.c_void_p
        L.refgpu_create.restype = vp
        L.refgpu_create.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.refgpu_destroy.argtypes = [vp]
        L.refgpu_set_atoms.argtypes = [vp, vp, vp]
        L.refgpu_compute.argtypes = [vp, _f64p, _i32p, vp, vp, vp]
        L.refgpu_neighbors.argtypes = [vp, ctypes.c_int, _i32p, _i32p, ctypes.c_int]
        L.refgpu_neighbors_small.argtypes = [vp, ctypes.c_int, _i32p, _i32p, ctypes.c_int]
        for f in ("refgpu_set_atoms", "refgpu_compute", "refgpu_neighbors",
                  "refgpu_neighbors_small"):
            getattr(L, f).restype = ctypes.c_int
        _refgpu = L
    return _refgpu


class RefGpuModel:
    """The reference's own FP32 GPU NEP (src/gpumd_compat compiled for sm_100a).

    Device buffers are torch CUDA tensors; the reference copies them into its
    own GPU_Vectors (set_atoms) and evaluates with its legacy kernel sequence.
    """

    def __init__(self, path, n):
        self._h = refgpu_lib().refgpu_create(os.fsencode(path), int(n))
        self.n = int(n)

    def __del__(self):
        if getattr(self, "_h", None):
            refgpu_lib().refgpu_destroy(self._h)
            self._h = None

    def set_atoms(self, d_type, d_pos):
        if refgpu_lib().refgpu_set_atoms(self._h, ctypes.c_void_p(d_type.data_ptr()),
                                         ctypes.c_void_p(d_pos.data_ptr())):
            raise RuntimeError("reference set_atoms failed")

    def compute(self, h, pbc=(1, 1, 1), out=None):
        h = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(9))
        pbc = np.ascontiguousarray(pbc, dtype=np.int32)
        ptrs = [ctypes.c_void_p(t.data_ptr()) for t in out] if out else [None, None, None]
        if refgpu_lib().refgpu_compute(self._h, h, pbc, *ptrs):
            raise RuntimeError("reference compute failed")

    def neighbors(self, which, mn, small=False):
        nn = np.zeros(self.n, dtype=np.int32)
        nl = np.zeros(self.n * mn, dtype=np.int32)
        fn = refgpu_lib().refgpu_neighbors_small if small else refgpu_lib().refgpu_neighbors
        if fn(self._h, which, nn, nl, mn):
            raise RuntimeError("reference neighbour rows unavailable")
        nl = nl.reshape(self.n, mn)
        return [nl[i, :nn[i]].copy() for i in range(self.n)]
