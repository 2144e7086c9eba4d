"""Python binding of the nepx C ABI (include/nepx.h) over ctypes.

The engine is lib/libnepx.so (C++ host code + sm_100a CUDA kernels).  This
module only marshals pointers: device buffers are torch CUDA tensors, and
every call goes straight to the shared library.  There is no CPU fallback:
loading fails loudly when the library is missing.

    pot = Potential("nep.txt", max_atoms=4096)
    pe, force, virial = pot.compute(types, box_h, positions)   # torch CUDA tensors

Names follow the reference's potential interface (Potential::compute,
src/gpumd_compat/potential.cuh:82-88): types 0-based in potential-file order,
positions SoA (3, n) in Angstrom, virial (9, n) in the order
xx yy zz xy xz yz yx zx zy.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnepx.so")

NEPX_ACCUMULATE = 1
NEPX_SYNC_CHECK = 2

ERRORS = {1: "NEPX_ERR_ARG", 2: "NEPX_ERR_FILE", 3: "NEPX_ERR_UNSUPPORTED", 4: "NEPX_ERR_CUDA",
          5: "NEPX_ERR_CAPACITY", 6: "NEPX_ERR_OVERFLOW", 7: "NEPX_ERR_NONFINITE",
          8: "NEPX_ERR_BOX"}

# every symbol include/nepx.h declares (checked by tests/test_capi_symbols.py)
EXPORTED = ["nepx_create", "nepx_destroy", "nepx_last_error", "nepx_info", "nepx_compute",
            "nepx_notify_box_changed", "nepx_set_skin", "nepx_neighbors", "nepx_neighbor_stats",
            "nepx_md_create", "nepx_md_destroy", "nepx_md_last_error", "nepx_md_set_ensemble",
            "nepx_md_run", "nepx_md_get", "nepx_md_device_state", "nepx_profile",
            "nepx_md_run_async", "nepx_md_sync", "nepx_compute_noalloc", "nepx_compute_batch",
            "nepx_server_create", "nepx_server_destroy", "nepx_server_last_error",
            "nepx_server_submit", "nepx_server_poll", "nepx_server_wait", "nepx_server_drain",
            "nepx_server_stats", "nepx_set_precision", "nepx_md_run_segment",
            "nepx_md_set_barostat", "nepx_md_set_velocity", "nepx_md_compute_forces",
            "nepx_md_neighbor_info", "nepx_md_set_max_distance", "nepx_md_time",
            "nepx_md_enable_unwrapped", "nepx_md_get_unwrapped", "nepx_server_create_budget",
            "nepx_server_memory", "nepx_server_set_row_reuse", "nepx_server_rows",
            "nepx_get_tuning", "nepx_set_tuning"]
TUNING_FIELDS = ("filter_group", "fused_group", "fused_ctas_per_sm", "f12_group",
                 "gather_group", "fused_f12", "gather_ctas_per_sm")

PRECISIONS = {"fp32": 0, "mixed": 1, "mixed_bf16": 2}
ENSEMBLES = {"nve": 0, "nvt_ber": 1, "nvt_nhc": 2, "nvt_bdp": 3, "npt_ber": 4, "npt_scr": 5}
BAROSTATS = {"isotropic": 0, "anisotropic": 1, "triclinic": 2}
THERMO_COLUMNS = ["T", "KE", "PE", "sxx", "syy", "szz", "syz", "sxz", "sxy", "ax", "ay", "az",
                  "bx", "by", "bz", "cx", "cy", "cz", "velocity_factor", "box_factor"]


class NepxError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("%s: %s" % (ERRORS.get(code, code), message))
        self.code = code


class Box(ctypes.Structure):
    _fields_ = [("h", ctypes.c_double * 9), ("pbc", ctypes.c_int * 3)]


class StructDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("box", Box)]


class Request(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("box", Box), ("type", ctypes.c_void_p),
                ("pos", ctypes.c_void_p), ("md_steps", ctypes.c_int), ("dt_fs", ctypes.c_double),
                ("mass", ctypes.c_void_p), ("vel", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("pe", ctypes.c_void_p), ("force", ctypes.c_void_p), ("virial", ctypes.c_void_p),
                ("pos", ctypes.c_void_p), ("vel", ctypes.c_void_p), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


_lib = None


def build():
    import subprocess
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


def lib():
    """Load lib/libnepx.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("nepx engine library not built: %s (run make -C dmg-md_b200)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.nepx_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]
        L.nepx_destroy.argtypes = [vp]
        L.nepx_last_error.argtypes = [vp]
        L.nepx_last_error.restype = ctypes.c_char_p
        L.nepx_info.argtypes = [vp, ip, dp]
        L.nepx_compute.argtypes = [vp, ctypes.POINTER(Box), ctypes.c_int, vp, vp, vp, vp, vp,
                                   ctypes.c_uint, vp]
        L.nepx_notify_box_changed.argtypes = [vp]
        L.nepx_set_skin.argtypes = [vp, ctypes.c_double]
        L.nepx_neighbors.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, ctypes.c_int, vp]
        L.nepx_neighbor_stats.argtypes = [vp, ip, ip, ip, vp]
        L.nepx_md_create.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.POINTER(Box), vp,
                                     ctypes.POINTER(vp)]
        L.nepx_md_destroy.argtypes = [vp]
        L.nepx_md_last_error.argtypes = [vp]
        L.nepx_md_last_error.restype = ctypes.c_char_p
        L.nepx_md_set_ensemble.argtypes = [vp, ctypes.c_int, dp, ctypes.c_uint]
        L.nepx_md_set_barostat.argtypes = [vp, ctypes.c_int, dp, dp]
        # the thermo buffer goes as an address (one-step calls are a hot loop)
        L.nepx_md_run.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp]
        L.nepx_md_get.argtypes = [vp, dp, dp, dp, dp, dp, ctypes.POINTER(Box)]
        L.nepx_compute_noalloc.argtypes = [vp, ctypes.POINTER(Box), ctypes.c_int, vp, vp, vp, vp,
                                           vp, vp]
        L.nepx_md_run_async.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        L.nepx_md_sync.argtypes = [vp]
        L.nepx_profile.argtypes = [vp, ctypes.POINTER(Box), ctypes.c_int, vp, vp, vp, vp, vp,
                                   ctypes.c_int, dp, vp]
        L.nepx_md_device_state.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                           ctypes.POINTER(vp), ctypes.POINTER(vp),
                                           ctypes.POINTER(vp)]
        L.nepx_set_precision.argtypes = [vp, ctypes.c_int]
        L.nepx_get_tuning.argtypes = [vp, ip, ip]
        L.nepx_set_tuning.argtypes = [vp, ip]
        L.nepx_md_run_segment.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp,
                                          ctypes.c_int, ctypes.c_int]
        L.nepx_compute_batch.argtypes = [vp, ctypes.POINTER(StructDesc), ctypes.c_int, vp, vp, vp,
                                         vp, vp, ctypes.c_uint, vp]
        L.nepx_server_create.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
        L.nepx_server_destroy.argtypes = [vp]
        L.nepx_server_last_error.argtypes = [vp]
        L.nepx_server_last_error.restype = ctypes.c_char_p
        L.nepx_server_submit.argtypes = [vp, ctypes.POINTER(Request), ctypes.POINTER(Result),
                                         ctypes.POINTER(ctypes.c_longlong)]
        L.nepx_server_poll.argtypes = [vp, ctypes.c_longlong, ip, ip]
        L.nepx_server_wait.argtypes = [vp, ctypes.c_longlong, ip]
        L.nepx_server_drain.argtypes = [vp]
        L.nepx_server_stats.argtypes = [vp, dp]
        L.nepx_server_create_budget.argtypes = [vp, ctypes.c_double, ctypes.c_int,
                                                ctypes.POINTER(vp)]
        L.nepx_server_memory.argtypes = [vp, dp]
        L.nepx_server_set_row_reuse.argtypes = [vp, ctypes.c_int]
        L.nepx_server_rows.argtypes = [vp, dp]
        L.nepx_md_set_velocity.argtypes = [vp, dp]
        L.nepx_md_compute_forces.argtypes = [vp]
        L.nepx_md_neighbor_info.argtypes = [vp, ip, ip]
        L.nepx_md_set_max_distance.argtypes = [vp, ctypes.c_double]
        L.nepx_md_time.argtypes = [vp, dp]
        L.nepx_md_enable_unwrapped.argtypes = [vp]
        L.nepx_md_get_unwrapped.argtypes = [vp, dp]
        for name in EXPORTED:
            if name not in ("nepx_last_error", "nepx_md_last_error", "nepx_server_last_error"):
                getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def make_box(h, pbc=(1, 1, 1)):
    b = Box()
    flat = [float(v) for v in (h.reshape(-1).tolist() if hasattr(h, "reshape") else h)]
    if len(flat) != 9:
        raise ValueError("box needs 9 numbers")
    for k in range(9):
        b.h[k] = flat[k]
    for k in range(3):
        b.pbc[k] = int(pbc[k])
    return b


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Potential:
    """A NEP potential on the current CUDA device (one nepx handle)."""

    def __init__(self, path, max_atoms):
        self._h = ctypes.c_void_p()
        rc = lib().nepx_create(os.fsencode(path), int(max_atoms), ctypes.byref(self._h))
        if rc:
            raise NepxError(rc, lib().nepx_last_error(None).decode())
        info = (ctypes.c_int * 16)()
        rcs = (ctypes.c_double * 32)()
        lib().nepx_info(self._h, info, rcs)
        keys = ["version", "num_types", "zbl", "zbl_flexible", "n_max_r", "n_max_a", "basis_r",
                "basis_a", "L_max", "num_L", "dim", "H", "MN_r", "MN_a", "has_q", "typewise_zbl"]
        self.info = dict(zip(keys, list(info)))
        self.max_atoms = int(max_atoms)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nepx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise NepxError(rc, lib().nepx_last_error(self._h).decode())

    def compute(self, types, h, pos, pbc=(1, 1, 1), out=None, accumulate=False, sync_check=False,
                stream=None):
        """Energy (n,), force (3, n), virial (9, n) as float64 CUDA tensors."""
        import torch
        n = types.numel()
        if out is None:
            pe = torch.empty(n, dtype=torch.float64, device=pos.device)
            force = torch.empty(3, n, dtype=torch.float64, device=pos.device)
            virial = torch.empty(9, n, dtype=torch.float64, device=pos.device)
        else:
            pe, force, virial = out
        assert types.dtype == torch.int32 and pos.dtype == torch.float64
        assert types.is_contiguous() and pos.is_contiguous()
        flags = (NEPX_ACCUMULATE if accumulate else 0) | (NEPX_SYNC_CHECK if sync_check else 0)
        box = make_box(h, pbc)
        self._check(lib().nepx_compute(self._h, ctypes.byref(box), n, _ptr(types), _ptr(pos),
                                       _ptr(pe), _ptr(force), _ptr(virial), flags,
                                       _stream_ptr(stream)))
        return pe, force, virial

    def set_precision(self, mode):
        """"fp32" (default), "mixed" (the ANN on the tensor cores, FP16 operands
        with per-layer scaling) or "mixed_bf16" (BF16 operands)."""
        self._check(lib().nepx_set_precision(self._h, PRECISIONS[mode]))

    def tuning(self):
        """The force kernels' launch choices (dict of TUNING_FIELDS) and whether
        they are fixed yet (the autotuner runs at the first compute)."""
        v = (ctypes.c_int * len(TUNING_FIELDS))()
        tuned = ctypes.c_int(0)
        self._check(lib().nepx_get_tuning(self._h, v, ctypes.byref(tuned)))
        return dict(zip(TUNING_FIELDS, list(v))), bool(tuned.value)

    def set_tuning(self, **choices):
        """Fixes the launch choices (the current ones, updated by `choices`)
        for every later call: no autotuning runs."""
        cur, _ = self.tuning()
        for k in choices:
            if k not in cur:
                raise KeyError(k)
        cur.update(choices)
        v = (ctypes.c_int * len(TUNING_FIELDS))(*[int(cur[k]) for k in TUNING_FIELDS])
        self._check(lib().nepx_set_tuning(self._h, v))

    def compute_batch(self, structs, types, pos, out=None, accumulate=False, sync_check=False,
                      stream=None):
        """Independent structures in one call.

        structs: list of (n, h, pbc); types (T,) int32 and pos (3, T) float64
        CUDA tensors with the structures back to back.  Returns pe (T,),
        force (3, T), virial (9, T)."""
        import torch
        T = types.numel()
        descs = (StructDesc * len(structs))()
        for k, (n, h, pbc) in enumerate(structs):
            descs[k].n = int(n)
            descs[k].box = make_box(h, pbc)
        if out is None:
            pe = torch.empty(T, dtype=torch.float64, device=pos.device)
            force = torch.empty(3, T, dtype=torch.float64, device=pos.device)
            virial = torch.empty(9, T, dtype=torch.float64, device=pos.device)
        else:
            pe, force, virial = out
        assert types.dtype == torch.int32 and pos.dtype == torch.float64
        assert types.is_contiguous() and pos.is_contiguous()
        flags = (NEPX_ACCUMULATE if accumulate else 0) | (NEPX_SYNC_CHECK if sync_check else 0)
        self._check(lib().nepx_compute_batch(self._h, descs, len(structs), _ptr(types), _ptr(pos),
                                             _ptr(pe), _ptr(force), _ptr(virial), flags,
                                             _stream_ptr(stream)))
        return pe, force, virial

    def neighbors(self, which, n, stream=None):
        """Rows of the last compute as a list of CPU numpy arrays (ascending)."""
        import torch
        mn = self.info["MN_r"] if which == 0 else self.info["MN_a"]
        nn = torch.empty(n, dtype=torch.int32, device="cuda")
        nl = torch.empty(n, mn, dtype=torch.int32, device="cuda")
        self._check(lib().nepx_neighbors(self._h, which, n, _ptr(nn), _ptr(nl), mn,
                                         _stream_ptr(stream)))
        torch.cuda.synchronize()
        nn = nn.cpu().numpy()
        nl = nl.cpu().numpy()
        return [nl[i, :nn[i]].copy() for i in range(n)]

    def neighbor_counts(self, which, n, stream=None):
        """Row lengths (numpy int32) of the first n atoms of the last compute."""
        import torch
        mn = self.info["MN_r"] if which == 0 else self.info["MN_a"]
        nn = torch.empty(n, dtype=torch.int32, device="cuda")
        nl = torch.empty(n, mn, dtype=torch.int32, device="cuda")
        self._check(lib().nepx_neighbors(self._h, which, n, _ptr(nn), _ptr(nl), mn,
                                         _stream_ptr(stream)))
        torch.cuda.synchronize()
        return nn.cpu().numpy()

    def neighbor_stats(self, stream=None):
        r, a, v = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(lib().nepx_neighbor_stats(self._h, ctypes.byref(r), ctypes.byref(a),
                                              ctypes.byref(v), _stream_ptr(stream)))
        return r.value, a.value, v.value

    def profile(self, types, h, pos, reps=20, pbc=(1, 1, 1), stream=None):
        """Per-stage device ms: neighbour, descriptor, gather, total."""
        import torch
        n = types.numel()
        pe = torch.empty(n, dtype=torch.float64, device=pos.device)
        force = torch.empty(3, n, dtype=torch.float64, device=pos.device)
        virial = torch.empty(9, n, dtype=torch.float64, device=pos.device)
        ms = (ctypes.c_double * 4)()
        box = make_box(h, pbc)
        self._check(lib().nepx_profile(self._h, ctypes.byref(box), n, _ptr(types), _ptr(pos),
                                       _ptr(pe), _ptr(force), _ptr(virial), int(reps), ms,
                                       _stream_ptr(stream)))
        return dict(zip(["neighbor", "descriptor", "gather", "total"], list(ms)))

    def notify_box_changed(self):
        self._check(lib().nepx_notify_box_changed(self._h))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class MD:
    """Device-resident MD of one system (nepx_md_* of include/nepx.h).

    Host numpy inputs: types (n,), masses (n,) amu, positions (3, n) A,
    velocities (3, n) A/fs, box h (9,) row-major with cell vectors as columns.
    """

    def __init__(self, potential, types, masses, pos, vel, h, pbc=(1, 1, 1)):
        import numpy as np
        self.pot = potential
        self.n = len(types)
        t = np.ascontiguousarray(types, dtype=np.int32)
        m = np.ascontiguousarray(masses, dtype=np.float64)
        x = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1)
        box = make_box(h, pbc)
        self._h = ctypes.c_void_p()
        rc = lib().nepx_md_create(potential._h, self.n, t.ctypes.data_as(ctypes.c_void_p),
                                  m.ctypes.data_as(ctypes.c_void_p),
                                  x.ctypes.data_as(ctypes.c_void_p),
                                  v.ctypes.data_as(ctypes.c_void_p), ctypes.byref(box), None,
                                  ctypes.byref(self._h))
        if rc:
            raise NepxError(rc, "nepx_md_create failed")

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nepx_md_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise NepxError(rc, lib().nepx_md_last_error(self._h).decode())

    def set_ensemble(self, kind, T0=0.0, T1=None, Tdamp=100.0, p_gpa=0.0, bulk_gpa=0.0,
                     tau_p=1000.0, seed=12345678):
        import numpy as np
        T1 = T0 if T1 is None else T1
        params = np.array([T0, T1, Tdamp, p_gpa, bulk_gpa, tau_p], dtype=np.float64)
        self._check(lib().nepx_md_set_ensemble(self._h, ENSEMBLES[kind], _dp(params), seed))

    def set_barostat(self, coupling, pressure_gpa=None, modulus_gpa=None):
        """Pressure coupling of the NPT ensemble: "isotropic", "anisotropic"
        (xx yy zz) or "triclinic" (xx yy zz yz xz xy) targets and moduli in GPa."""
        import numpy as np
        code = BAROSTATS[coupling]
        if code == 0:
            self._check(lib().nepx_md_set_barostat(self._h, 0, None, None))
            return
        pr = np.ascontiguousarray(pressure_gpa, dtype=np.float64)
        mo = np.ascontiguousarray(modulus_gpa, dtype=np.float64)
        if pr.size != (3 if code == 1 else 6) or mo.size != pr.size:
            raise ValueError("%s coupling takes %d pressures and moduli"
                             % (coupling, 3 if code == 1 else 6))
        self._check(lib().nepx_md_set_barostat(self._h, code, _dp(pr), _dp(mo)))

    def run(self, steps, dt_fs, thermo_every=0):
        """Runs `steps` steps; returns the thermo rows (rows, 20) or None."""
        import numpy as np
        rows = steps // thermo_every if thermo_every else 0
        out = np.zeros((max(rows, 1), len(THERMO_COLUMNS)))
        self._check(lib().nepx_md_run(self._h, steps, dt_fs, thermo_every,
                                      out.ctypes.data if rows else None))
        return out[:rows] if rows else None

    def run_segment(self, steps, dt_fs, first_step, segment_steps, thermo_every=0):
        """Steps [first_step, first_step + steps) of a segment of segment_steps."""
        import numpy as np
        rows = steps // thermo_every if thermo_every else 0
        out = np.zeros((max(rows, 1), len(THERMO_COLUMNS)))
        self._check(lib().nepx_md_run_segment(self._h, steps, dt_fs, thermo_every,
                                              out.ctypes.data if rows else None, first_step,
                                              segment_steps))
        return out[:rows] if rows else None

    def run_async(self, steps, dt_fs):
        self._check(lib().nepx_md_run_async(self._h, steps, dt_fs))

    def set_velocity(self, vel):
        """Replaces the velocities, (3, n) A/fs."""
        import numpy as np
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1)
        self._check(lib().nepx_md_set_velocity(self._h, _dp(v)))

    def compute_forces(self):
        """Energy, forces and virials at the current positions."""
        self._check(lib().nepx_md_compute_forces(self._h))

    def neighbor_info(self):
        """(largest radial row, largest angular row) of the latest force evaluation."""
        r, a = ctypes.c_int(), ctypes.c_int()
        self._check(lib().nepx_md_neighbor_info(self._h, ctypes.byref(r), ctypes.byref(a)))
        return r.value, a.value

    def set_max_distance(self, max_distance):
        """Adaptive time step bound in A (0: fixed step)."""
        self._check(lib().nepx_md_set_max_distance(self._h, float(max_distance)))

    def time(self):
        """Simulated time (fs) since the current segment's first step."""
        t = ctypes.c_double()
        self._check(lib().nepx_md_time(self._h, ctypes.byref(t)))
        return t.value

    def enable_unwrapped(self):
        self._check(lib().nepx_md_enable_unwrapped(self._h))

    def unwrapped(self):
        """Unwrapped positions (3, n) in A."""
        import numpy as np
        out = np.zeros((3, self.n))
        self._check(lib().nepx_md_get_unwrapped(self._h, _dp(out)))
        return out

    def sync(self):
        self._check(lib().nepx_md_sync(self._h))

    def device_state(self):
        """(d_pos, d_vel, d_force, d_type, stream) raw pointers."""
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        self._check(lib().nepx_md_device_state(self._h, *[ctypes.byref(p) for p in ptrs]))
        return [p.value for p in ptrs]

    def state(self):
        import numpy as np
        n = self.n
        pos, vel, force = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n)
        pe, vir = np.zeros(n), np.zeros(9 * n)
        box = Box()
        self._check(lib().nepx_md_get(self._h, _dp(pos), _dp(vel), _dp(force), _dp(pe),
                                      _dp(vir), ctypes.byref(box)))
        return {"pos": pos.reshape(3, n), "vel": vel.reshape(3, n), "force": force.reshape(3, n),
                "pe": pe, "virial": vir.reshape(9, n), "h": np.array(box.h[:])}


class Server:
    """Continuous-batching server over one potential (nepx_server_* of include/nepx.h).

    submit() copies a request (host numpy arrays) and returns a ticket; the
    results land in numpy arrays owned by this object once wait()/poll()
    report the ticket done."""

    def __init__(self, potential, max_atoms=None, max_struct=2048, hbm_bytes=None):
        """An arena of max_atoms atoms, or one sized from a device-memory
        budget (hbm_bytes) that admission then holds to."""
        self.pot = potential
        self._h = ctypes.c_void_p()
        if hbm_bytes is not None:
            rc = lib().nepx_server_create_budget(potential._h, float(hbm_bytes), int(max_struct),
                                                 ctypes.byref(self._h))
        else:
            rc = lib().nepx_server_create(potential._h, int(max_atoms), int(max_struct),
                                          ctypes.byref(self._h))
        if rc:
            raise NepxError(rc, lib().nepx_last_error(potential._h).decode())
        self._out = {}

    def memory(self):
        """budget_bytes, bytes_per_atom, bytes_per_struct, mean_resident_bytes."""
        info = (ctypes.c_double * 4)()
        self._check(lib().nepx_server_memory(self._h, info))
        keys = ["budget_bytes", "bytes_per_atom", "bytes_per_struct", "mean_resident_bytes"]
        return dict(zip(keys, list(info)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nepx_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise NepxError(rc, lib().nepx_server_last_error(self._h).decode())

    def submit(self, types, pos, h, pbc=(1, 1, 1), md_steps=0, dt_fs=0.0, masses=None, vel=None,
               want_virial=True, want_state=False):
        import numpy as np
        n = len(types)
        keep = {"type": np.ascontiguousarray(types, dtype=np.int32),
                "pos_in": np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)}
        req = Request()
        req.n = n
        req.box = make_box(h, pbc)
        req.type = keep["type"].ctypes.data
        req.pos = keep["pos_in"].ctypes.data
        req.md_steps = int(md_steps)
        req.dt_fs = float(dt_fs)
        if md_steps:
            keep["mass"] = np.ascontiguousarray(masses, dtype=np.float64)
            keep["vel_in"] = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1)
            req.mass = keep["mass"].ctypes.data
            req.vel = keep["vel_in"].ctypes.data
        res = Result()
        keep["pe"] = np.zeros(n)
        keep["force"] = np.zeros((3, n))
        res.pe = keep["pe"].ctypes.data
        res.force = keep["force"].ctypes.data
        if want_virial:
            keep["virial"] = np.zeros((9, n))
            res.virial = keep["virial"].ctypes.data
        if want_state:
            keep["pos"] = np.zeros((3, n))
            keep["vel"] = np.zeros((3, n))
            res.pos = keep["pos"].ctypes.data
            res.vel = keep["vel"].ctypes.data
        keep["result"] = res
        ticket = ctypes.c_longlong()
        self._check(lib().nepx_server_submit(self._h, ctypes.byref(req), ctypes.byref(res),
                                             ctypes.byref(ticket)))
        self._out[ticket.value] = keep
        return ticket.value

    def poll(self, ticket):
        done, status = ctypes.c_int(), ctypes.c_int()
        self._check(lib().nepx_server_poll(self._h, ticket, ctypes.byref(done),
                                           ctypes.byref(status)))
        return bool(done.value)

    def wait(self, ticket):
        """Blocks until the ticket is done; returns its results (dict of numpy arrays)."""
        status = ctypes.c_int()
        self._check(lib().nepx_server_wait(self._h, ticket, ctypes.byref(status)))
        if status.value:
            raise NepxError(status.value, lib().nepx_server_last_error(self._h).decode())
        keep = self._out.pop(ticket)
        r = keep["result"]
        out = {k: keep[k] for k in ("pe", "force", "virial", "pos", "vel") if k in keep}
        out.update(t_submit=r.t_submit, t_admit=r.t_admit, t_done=r.t_done)
        return out

    def drain(self):
        self._check(lib().nepx_server_drain(self._h))

    def set_row_reuse(self, on):
        """Row reuse (Verlet candidates) for MD segments admitted from now on."""
        self._check(lib().nepx_server_set_row_reuse(self._h, 1 if on else 0))

    def rows(self):
        """{'builds': centers whose candidates were built, 'kept': centers of
        candidate-keeping structures summed over the steps}."""
        s = (ctypes.c_double * 2)()
        self._check(lib().nepx_server_rows(self._h, s))
        return {"builds": s[0], "kept": s[1]}

    def stats(self):
        s = (ctypes.c_double * 8)()
        self._check(lib().nepx_server_stats(self._h, s))
        keys = ["done", "steps", "atom_steps", "busy_s", "mean_atoms", "mean_structs", "queued",
                "uptime_s"]
        return dict(zip(keys, list(s)))
