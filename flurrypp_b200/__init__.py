"""B200 Flux Reconstruction residual and RK update (FlurryPP's solver path).

Python binding of ``libfr_b200.so`` (C ABI in ``include/fr_b200.h``).  The
``Solver`` class mirrors the reference ``solver`` interface
(``include/solver.hpp:147-178``): it is set up from a reference input deck,
``calc_residual(step)`` fills ``divF_spts[step]`` and ``update()`` advances one
time step.  State arrays keep the reference layout
``[point][element][field]``.

The compute path is the CUDA library only: if ``libfr_b200.so`` is missing or
does not load, importing :mod:`flurrypp_b200` raises.
"""
from __future__ import annotations

import ctypes
import os

# Hardware work queues per process: CUDA's default of 8 makes streams beyond
# the eighth share queues, which serialises the per-request streams of the
# server (measured: 16 channel solves in flight, 0.63 -> 0.69 solves/s FP64,
# 0.66 -> 0.93 in the precision form).  Takes effect only if set before the
# process creates its CUDA context; a value the caller set is kept.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfr_b200.so")

FR_OK = 0
FR_ERR_ARG = 1
FR_ERR_SETUP = 2
FR_ERR_CUDA = 3
FR_ERR_NONFINITE = 4
FR_ERR_BUDGET = 5
FR_ERR_TIMEOUT = 6
FR_ERR_UNSUPPORTED = 7
FR_ERR_STATE = 8

FR_BATCH_GROUPS, FR_BATCH_MANY_ORDER = 0, 1
FR_PREC_FP64 = 0
FR_PREC_MIXED = 1
FR_PREC_MIXED_REFINE = 2  # server: precision form until the FP32 floor, then FP64 to the target

IC_DECK, IC_VORTEX, IC_TGV, IC_UNIFORM = 0, 1, 2, 3


class FrError(RuntimeError):
    """A non-zero status from the library, with its message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[fr status {code}] {msg}")
        self.code = code


class SetupOpts(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int),
        ("perturb", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("perturb_frac", ctypes.c_double),
        ("mu_override", ctypes.c_int),
        ("mu_inf", ctypes.c_double),
        ("visc_flux_quirk", ctypes.c_int),
        ("debug_arrays", ctypes.c_int),
        ("device", ctypes.c_int),
        ("generic_kernels", ctypes.c_int),
        ("no_tma", ctypes.c_int),
        ("tile_variant", ctypes.c_int),
        ("no_tensor_cores", ctypes.c_int),
        ("no_pdl", ctypes.c_int),
    ]


class Mesh(ctypes.Structure):
    _fields_ = [
        ("nDims", ctypes.c_int),
        ("nVerts", ctypes.c_int),
        ("xv", ctypes.POINTER(ctypes.c_double)),
        ("nEles", ctypes.c_int),
        ("nNodes", ctypes.c_int),
        ("c2v", ctypes.POINTER(ctypes.c_int)),
        ("nBndFaces", ctypes.c_int),
        ("bndFaceVerts", ctypes.POINTER(ctypes.c_int)),
        ("bndFaceBc", ctypes.POINTER(ctypes.c_int)),
        ("period", ctypes.c_double * 3),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("nDims", ctypes.c_int),
        ("nFields", ctypes.c_int),
        ("order", ctypes.c_int),
        ("nEles", ctypes.c_int),
        ("nSpts", ctypes.c_int),
        ("nFpts", ctypes.c_int),
        ("nFaces", ctypes.c_int),
        ("nFacePts", ctypes.c_int),
        ("nRKSteps", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("dtType", ctypes.c_int),
        ("timeType", ctypes.c_int),
        ("iter", ctypes.c_longlong),
        ("time", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("tensor_kernels", ctypes.c_int),
        ("tile_variant", ctypes.c_int),
        ("elems_per_block", ctypes.c_int),
    ]


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i = ctypes.c_int
    dp = ctypes.POINTER(ctypes.c_double)
    sz = ctypes.c_size_t
    sigs = {
        "fr_setup_opts_default": (None, [ctypes.POINTER(SetupOpts)]),
        "fr_create_from_deck": (i, [ctypes.c_char_p, ctypes.POINTER(SetupOpts), ctypes.POINTER(P)]),
        "fr_create_with_mesh": (i, [ctypes.c_char_p, ctypes.POINTER(Mesh), ctypes.POINTER(SetupOpts), ctypes.POINTER(P)]),
        "fr_destroy": (None, [P]),
        "fr_last_error": (ctypes.c_char_p, [P]),
        "fr_get_info": (i, [P, ctypes.POINTER(Info)]),
        "fr_set_stream": (i, [P, P]),
        "fr_init_solution": (i, [P, i, dp, i]),
        "fr_set_state": (i, [P, dp, sz]),
        "fr_get_state": (i, [P, dp, sz]),
        "fr_get_state_async": (i, [P, dp, sz]),
        "fr_calc_residual": (i, [P, i]),
        "fr_get_residual": (i, [P, i, dp, sz]),
        "fr_update": (i, [P, i]),
        "fr_run": (i, [P, i]),
        "fr_pmg_cycle": (i, [P]),
        "fr_calc_dt": (i, [P, dp]),
        "fr_set_dt": (i, [P, ctypes.c_double]),
        "fr_residual_norm": (i, [P, i, dp, i]),
        "fr_check_state": (i, [P]),
        "fr_get_array": (i, [P, ctypes.c_char_p, P, ctypes.POINTER(sz)]),
        "fr_device_ptr": (i, [P, ctypes.c_char_p, ctypes.POINTER(P), ctypes.POINTER(sz)]),
        "fr_synchronize": (i, [P]),
        "fr_checkpoint": (i, [P]),
        "fr_integrate_error": (i, [P, i, dp, i]),
        "fr_wall_force": (i, [P, dp]),
        "fr_mass_flux": (i, [P, i, dp, i]),
        "fr_shard_plan": (i, [P, i, i, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong),
                              ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong]),
        "fr_write_data": (i, [P, ctypes.c_char_p]),
        "fr_read_restart": (i, [P, ctypes.c_char_p]),
        "fr_bench_kernel": (i, [P, ctypes.c_char_p, i]),
        "fr_batch_create": (i, [ctypes.POINTER(P), i, ctypes.POINTER(P)]),
        "fr_batch_run": (i, [P, i]),
        "fr_batch_gather": (i, [P]),
        "fr_batch_residual_norms": (i, [P, i, dp, i]),
        "fr_batch_info": (i, [P, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong)]),
        "fr_batch_last_error": (ctypes.c_char_p, [P]),
        "fr_batch_form": (i, [P, ctypes.POINTER(i), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
        "fr_batch_set_form": (i, [P, i]),
        "fr_batch_destroy": (None, [P]),
        "fr_server_create": (i, [sz, i, i, i, ctypes.POINTER(P)]),
        "fr_server_submit": (i, [P, ctypes.c_char_p, ctypes.POINTER(Mesh), i, dp, i, ctypes.c_double, i,
                                 ctypes.POINTER(ctypes.c_longlong)]),
        "fr_server_poll": (i, [P, ctypes.c_longlong, ctypes.POINTER(i), dp, ctypes.POINTER(i), dp]),
        "fr_server_wait": (i, [P, ctypes.c_longlong, ctypes.c_double]),
        "fr_server_poll_form": (i, [P, ctypes.c_longlong, ctypes.POINTER(i), ctypes.POINTER(i)]),
        "fr_server_result": (i, [P, ctypes.c_longlong, dp, sz]),
        "fr_server_cancel": (i, [P, ctypes.c_longlong]),
        "fr_server_stats": (i, [P, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(sz)]),
        "fr_server_destroy": (None, [P]),
        "fr_server_set_precision": (i, [P, i]),
        "fr_shard_create": (i, [ctypes.c_char_p, ctypes.POINTER(SetupOpts), i, ctypes.POINTER(P)]),
        "fr_part_create": (i, [ctypes.c_char_p, ctypes.POINTER(SetupOpts), i, i, P, ctypes.POINTER(P)]),
        "fr_part_nccl_ok": (i, [P]),
        "fr_nccl_unique_id": (i, [ctypes.c_char_p]),
        "fr_nccl_comm_init": (i, [i, ctypes.c_char_p, i, i, ctypes.POINTER(P)]),
        "fr_nccl_comm_destroy": (i, [P]),
        "fr_shard_info": (i, [P, ctypes.POINTER(i), ctypes.POINTER(i), ctypes.POINTER(ctypes.c_longlong)]),
        "fr_shard_set_state": (i, [P, dp, sz]),
        "fr_shard_get_state": (i, [P, dp, sz]),
        "fr_shard_set_dt": (i, [P, ctypes.c_double]),
        "fr_shard_calc_residual": (i, [P, i]),
        "fr_shard_get_residual": (i, [P, i, dp, sz]),
        "fr_shard_run": (i, [P, i]),
        "fr_shard_time": (i, [P, dp, dp]),
        "fr_shard_last_error": (ctypes.c_char_p, [P]),
        "fr_shard_destroy": (None, [P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def default_opts(**kw) -> SetupOpts:
    o = SetupOpts()
    lib.fr_setup_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Solver:
    """One FR case on the GPU (the reference ``solver`` + its ``input``)."""

    def __init__(self, deck: str, mesh: dict | None = None, part=None, **opts):
        """part = (nparts, rank, nccl_comm): this rank's part of the case split
        by the partition of shard_plan (fr_part_create)."""
        self._c = ctypes.c_void_p()
        o = default_opts(**opts)
        if part is not None:
            nparts, rank, comm = part
            st = lib.fr_part_create(deck.encode(), ctypes.byref(o), nparts, rank, comm, ctypes.byref(self._c))
        elif mesh is None:
            st = lib.fr_create_from_deck(deck.encode(), ctypes.byref(o), ctypes.byref(self._c))
        else:
            self._mesh_keep = m = _make_mesh(mesh)
            st = lib.fr_create_with_mesh(deck.encode(), ctypes.byref(m[0]), ctypes.byref(o), ctypes.byref(self._c))
        if st != FR_OK:
            msg = lib.fr_last_error(self._c).decode() if self._c else "allocation failed"
            lib.fr_destroy(self._c)
            self._c = None
            raise FrError(st, msg)
        inf = self.info()
        self.nDims, self.nFields, self.order = inf.nDims, inf.nFields, inf.order
        self.nEles, self.nSpts, self.nFpts = inf.nEles, inf.nSpts, inf.nFpts
        self.nRKSteps = inf.nRKSteps
        self.shape = (self.nSpts, self.nEles, self.nFields)

    def __del__(self):
        if getattr(self, "_c", None):
            lib.fr_destroy(self._c)
            self._c = None

    def close(self):
        self.__del__()

    def _check(self, st: int):
        if st != FR_OK:
            raise FrError(st, lib.fr_last_error(self._c).decode())

    def info(self) -> Info:
        inf = Info()
        self._check(lib.fr_get_info(self._c, ctypes.byref(inf)))
        return inf

    def initialize_solution(self, kind: int = IC_DECK, prm=()):
        p = np.ascontiguousarray(prm, dtype=np.float64)
        self._check(lib.fr_init_solution(self._c, kind, _dptr(p) if p.size else None, int(p.size)))

    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(lib.fr_set_state(self._c, _dptr(U), U.size))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        """U_spts [nSpts, nEles, nFields]; into `out` (e.g. pinned host
        memory, C-contiguous float64 of that shape) when given."""
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        elif out.dtype != np.float64 or out.size != self.nSpts * self.nEles * self.nFields or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of the state's size")
        self._check(lib.fr_get_state(self._c, _dptr(out), out.size))
        return out

    def get_state_async(self, out: np.ndarray) -> np.ndarray:
        """Queue the copy of U_spts into `out` (pinned, C-contiguous float64)
        on the case's stream; valid once that stream has reached it."""
        if out.dtype != np.float64 or out.size != self.nSpts * self.nEles * self.nFields or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of the state's size")
        self._check(lib.fr_get_state_async(self._c, _dptr(out), out.size))
        return out

    def calc_residual(self, step: int = 0):
        self._check(lib.fr_calc_residual(self._c, step))

    def get_residual(self, step: int = 0) -> np.ndarray:
        d = np.empty(self.shape, dtype=np.float64)
        self._check(lib.fr_get_residual(self._c, step, _dptr(d), d.size))
        return d

    def update(self, pmg_source: bool = False):
        self._check(lib.fr_update(self._c, int(pmg_source)))

    def run(self, nsteps: int):
        """nsteps of update() (+ the P-multigrid cycle with PMG 1)."""
        self._check(lib.fr_run(self._c, nsteps))

    def pmg_cycle(self):
        self._check(lib.fr_pmg_cycle(self._c))

    def integrate_error(self, error_norm: int = -1) -> np.ndarray:
        """integrateError of the deck's test case (errorNorm 0, 1, 2; -1: deck's)."""
        out = np.zeros(self.nFields)
        self._check(lib.fr_integrate_error(self._c, int(error_norm), _dptr(out), self.nFields))
        return out

    def wall_force(self) -> np.ndarray:
        """writeResidual's force coefficients: pressure (x, y, z), viscous (x, y, z)."""
        out = np.zeros(6)
        self._check(lib.fr_wall_force(self._c, _dptr(out)))
        return out

    def mass_flux(self, error_norm: int = -1) -> np.ndarray:
        """computeMassFlux (testCase 2 monitor) per field."""
        out = np.zeros(self.nFields)
        self._check(lib.fr_mass_flux(self._c, int(error_norm), _dptr(out), self.nFields))
        return out

    def shard_plan(self, nparts: int, rank: int):
        """Sharding plan for part `rank` of `nparts` (host only; see
        fr_shard_plan): (part of every element, owned element count, halo
        peers, halo slots), the halo in the order both sides of a cut share."""
        part = np.zeros(self.nEles, dtype=np.int32)
        n_owned, n_halo = ctypes.c_int(0), ctypes.c_longlong(0)
        ip = ctypes.POINTER(ctypes.c_int)
        lp = ctypes.POINTER(ctypes.c_longlong)
        self._check(lib.fr_shard_plan(self._c, int(nparts), int(rank), part.ctypes.data_as(ip),
                                      ctypes.byref(n_owned), ctypes.byref(n_halo), None, None, 0))
        peer = np.zeros(n_halo.value, dtype=np.int32)
        slot = np.zeros(n_halo.value, dtype=np.int64)
        if n_halo.value:
            self._check(lib.fr_shard_plan(self._c, int(nparts), int(rank), None, ctypes.byref(n_owned),
                                          ctypes.byref(n_halo), peer.ctypes.data_as(ip), slot.ctypes.data_as(lp),
                                          n_halo.value))
        return part, n_owned.value, peer, slot

    def checkpoint(self):
        """Snapshot for output; the copy to the host overlaps later steps."""
        self._check(lib.fr_checkpoint(self._c))

    def write_data(self, path: str | None = None):
        """writeData: ParaView .vtu (plotType 1) or CSV (plotType 0)."""
        self._check(lib.fr_write_data(self._c, path.encode() if path else None))

    def read_restart(self, path: str | None = None):
        """readRestartFile: state and time from a .vtu (deck name if None)."""
        self._check(lib.fr_read_restart(self._c, path.encode() if path else None))

    def calc_dt(self) -> float:
        d = ctypes.c_double()
        self._check(lib.fr_calc_dt(self._c, ctypes.byref(d)))
        return d.value

    def set_dt(self, dt: float):
        self._check(lib.fr_set_dt(self._c, float(dt)))

    def residual_norm(self, res_type: int = 2) -> np.ndarray:
        out = np.empty(self.nFields, dtype=np.float64)
        self._check(lib.fr_residual_norm(self._c, res_type, _dptr(out), self.nFields))
        return out

    def check_state(self):
        self._check(lib.fr_check_state(self._c))

    def synchronize(self):
        self._check(lib.fr_synchronize(self._c))

    def get_array(self, name: str) -> np.ndarray:
        n = ctypes.c_size_t(0)
        self._check(lib.fr_get_array(self._c, name.encode(), None, ctypes.byref(n)))
        dt = np.int32 if name.startswith("face_") else np.float64
        a = np.empty(n.value, dtype=dt)
        self._check(lib.fr_get_array(self._c, name.encode(), a.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n)))
        return a

    def set_stream(self, stream_handle: int):
        """Run this case's kernels on a given cudaStream_t (e.g. torch's)."""
        self._check(lib.fr_set_stream(self._c, ctypes.c_void_p(stream_handle)))

    def bench_kernel(self, kernel: str, reps: int):
        self._check(lib.fr_bench_kernel(self._c, kernel.encode(), reps))

    def device_ptr(self, name: str):
        p = ctypes.c_void_p()
        b = ctypes.c_size_t()
        self._check(lib.fr_device_ptr(self._c, name.encode(), ctypes.byref(p), ctypes.byref(b)))
        return p.value, b.value


def nccl_comm(nranks: int, rank: int, device: int, unique_id: bytes | None = None):
    """An NCCL communicator through the library (fr_nccl_*): rank 0 passes
    unique_id=None and shares the returned id with the others, which pass it.
    Returns (comm, id)."""
    idb = ctypes.create_string_buffer(128)
    if unique_id is None:
        st = lib.fr_nccl_unique_id(idb)
        if st != FR_OK:
            raise FrError(st, "ncclGetUniqueId")
    else:
        ctypes.memmove(idb, unique_id, 128)
    comm = ctypes.c_void_p()
    st = lib.fr_nccl_comm_init(nranks, idb, rank, device, ctypes.byref(comm))
    if st != FR_OK:
        raise FrError(st, "ncclCommInitRank")
    return comm, idb.raw


class Shard:
    """One case split into `nparts` parts on one device (fr_shard_*): the
    partition of Solver.shard_plan, the cut faces' traces exchanged between
    the parts at every stage.  State and residual in the whole case's layout."""

    def __init__(self, deck: str, nparts: int, **opts):
        o = default_opts(**opts)
        self._s = ctypes.c_void_p()
        st = lib.fr_shard_create(deck.encode(), ctypes.byref(o), nparts, ctypes.byref(self._s))
        if st != FR_OK:
            msg = lib.fr_shard_last_error(self._s).decode() if self._s else "shard create failed"
            lib.fr_shard_destroy(self._s)
            self._s = None
            raise FrError(st, msg)
        self.nparts = nparts
        self.host = Solver(deck, device=-1, **{k: v for k, v in opts.items() if k != "device"})
        self.shape = self.host.shape

    def __del__(self):
        if getattr(self, "_s", None):
            lib.fr_shard_destroy(self._s)
            self._s = None

    def _check(self, st):
        if st != FR_OK:
            raise FrError(st, lib.fr_shard_last_error(self._s).decode())

    def info(self):
        n = ctypes.c_int()
        owned = (ctypes.c_int * self.nparts)()
        cut = (ctypes.c_longlong * self.nparts)()
        self._check(lib.fr_shard_info(self._s, ctypes.byref(n), owned, cut))
        return {"nparts": n.value, "owned": list(owned), "cut_points": list(cut)}

    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(lib.fr_shard_set_state(self._s, _dptr(U), U.size))

    def get_state(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(lib.fr_shard_get_state(self._s, _dptr(out), out.size))
        return out

    def set_dt(self, dt: float):
        self._check(lib.fr_shard_set_dt(self._s, dt))

    def calc_residual(self, step: int = 0):
        self._check(lib.fr_shard_calc_residual(self._s, step))

    def get_residual(self, step: int = 0) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(lib.fr_shard_get_residual(self._s, step, _dptr(out), out.size))
        return out

    def run(self, nsteps: int):
        self._check(lib.fr_shard_run(self._s, nsteps))

    def time(self):
        t, d = ctypes.c_double(), ctypes.c_double()
        self._check(lib.fr_shard_time(self._s, ctypes.byref(t), ctypes.byref(d)))
        return t.value, d.value


class Batch:
    """Many independent cases advanced together (fr_batch_*): same-order cases
    merged into one group, one face + one element launch per stage per order."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s._c.value for s in self.solvers])
        self._b = ctypes.c_void_p()
        st = lib.fr_batch_create(arr, len(self.solvers), ctypes.byref(self._b))
        if st != FR_OK:
            msg = lib.fr_batch_last_error(self._b).decode() if self._b else "batch create failed"
            lib.fr_batch_destroy(self._b)
            self._b = None
            raise FrError(st, msg)

    def __del__(self):
        if getattr(self, "_b", None):
            lib.fr_batch_destroy(self._b)
            self._b = None

    def _check(self, st):
        if st != FR_OK:
            raise FrError(st, lib.fr_batch_last_error(self._b).decode())

    def run(self, nsteps: int):
        self._check(lib.fr_batch_run(self._b, nsteps))

    def gather(self):
        """Copy every member's state (and last stage-0 residual) back to its case."""
        self._check(lib.fr_batch_gather(self._b))

    def residual_norms(self, res_type: int = 2) -> np.ndarray:
        nf = self.solvers[0].nFields
        out = np.empty((len(self.solvers), nf), dtype=np.float64)
        self._check(lib.fr_batch_residual_norms(self._b, res_type, _dptr(out), nf))
        return out

    def form(self) -> dict:
        """The step form in use (FR_BATCH_GROUPS / FR_BATCH_MANY_ORDER) and the
        ms per step each form measured at creation (-1: not timed)."""
        f, a, b = ctypes.c_int(), ctypes.c_float(), ctypes.c_float()
        self._check(lib.fr_batch_form(self._b, ctypes.byref(f), ctypes.byref(a), ctypes.byref(b)))
        return {"form": f.value, "ms_groups": a.value, "ms_many_order": b.value}

    def set_form(self, form: int):
        self._check(lib.fr_batch_set_form(self._b, form))

    def info(self):
        g = ctypes.c_int()
        n = ctypes.c_longlong()
        self._check(lib.fr_batch_info(self._b, ctypes.byref(g), ctypes.byref(n)))
        return {"groups": g.value, "launches": n.value}


class Server:
    """Continuous-batching solve server (fr_server_*)."""

    def __init__(self, budget_bytes: int, max_inflight: int = 8, check_every: int = 10, device: int = 0,
                 precision: int = FR_PREC_FP64):
        self._s = ctypes.c_void_p()
        st = lib.fr_server_create(int(budget_bytes), max_inflight, check_every, device, ctypes.byref(self._s))
        if st != FR_OK:
            raise FrError(st, "server create failed")
        st = lib.fr_server_set_precision(self._s, int(precision))
        if st != FR_OK:
            raise FrError(st, "server precision")
        self._keep = {}

    def close(self):
        if getattr(self, "_s", None):
            lib.fr_server_destroy(self._s)
            self._s = None

    __del__ = close

    def submit(self, deck: str, mesh: dict | None = None, ic=(IC_DECK, ()), tol: float = 1e-8,
               max_steps: int = 100000) -> int:
        kind, prm = ic
        p = np.ascontiguousarray(prm, dtype=np.float64)
        m = _make_mesh(mesh) if mesh is not None else None
        rid = ctypes.c_longlong()
        st = lib.fr_server_submit(self._s, deck.encode(), ctypes.byref(m[0]) if m else None, kind,
                                  _dptr(p) if p.size else None, int(p.size), tol, max_steps, ctypes.byref(rid))
        if st != FR_OK:
            raise FrError(st, "submit failed")
        return rid.value

    def poll(self, rid: int) -> dict:
        stt, steps = ctypes.c_int(), ctypes.c_int()
        lat, ratio = ctypes.c_double(), ctypes.c_double()
        code = lib.fr_server_poll(self._s, rid, ctypes.byref(stt), ctypes.byref(lat), ctypes.byref(steps),
                                  ctypes.byref(ratio))
        return {"status": stt.value, "latency_s": lat.value, "steps": steps.value, "res_ratio": ratio.value,
                "code": code}

    def poll_form(self, rid: int) -> dict:
        """Form the request runs in and its steps in the precision form."""
        prec, n32 = ctypes.c_int(), ctypes.c_int()
        st = lib.fr_server_poll_form(self._s, rid, ctypes.byref(prec), ctypes.byref(n32))
        if st != FR_OK:
            raise FrError(st, "poll_form failed")
        return {"precision": prec.value, "steps_fp32": n32.value}

    def wait(self, rid: int, timeout_s: float = 600.0):
        st = lib.fr_server_wait(self._s, rid, timeout_s)
        if st != FR_OK:
            raise FrError(st, f"request {rid} did not finish cleanly")

    def result(self, rid: int, shape) -> np.ndarray:
        U = np.empty(shape, dtype=np.float64)
        st = lib.fr_server_result(self._s, rid, _dptr(U), U.size)
        if st != FR_OK:
            raise FrError(st, "no result")
        return U

    def cancel(self, rid: int):
        lib.fr_server_cancel(self._s, rid)

    def stats(self) -> dict:
        q, f = ctypes.c_int(), ctypes.c_int()
        b = ctypes.c_size_t()
        lib.fr_server_stats(self._s, ctypes.byref(q), ctypes.byref(f), ctypes.byref(b))
        return {"queued": q.value, "inflight": f.value, "inflight_bytes": b.value}


def _make_mesh(m: dict):
    xv = np.ascontiguousarray(m["xv"], dtype=np.float64)
    c2v = np.ascontiguousarray(m["c2v"], dtype=np.int32)
    bfv = np.ascontiguousarray(m["bnd_face_verts"], dtype=np.int32).reshape(-1, 4)
    bfb = np.ascontiguousarray(m["bnd_face_bc"], dtype=np.int32)
    M = Mesh()
    M.nDims = int(xv.shape[1])
    M.nVerts = int(xv.shape[0])
    M.xv = xv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    M.nEles = int(c2v.shape[0])
    M.nNodes = int(c2v.shape[1])
    M.c2v = c2v.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    M.nBndFaces = int(bfb.size)
    M.bndFaceVerts = bfv.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    M.bndFaceBc = bfb.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    per = m.get("period", (1e300, 1e300, 1e300))
    for d in range(3):
        M.period[d] = float(per[d])
    return (M, xv, c2v, bfv, bfb)
