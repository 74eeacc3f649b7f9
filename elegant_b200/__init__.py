"""elegant_b200: B200 particle tracking for elegant's do_tracking() path.

A thin ctypes layer over libtrkgpu.so (C ABI in include/trk.h).  Python is
the test and benchmark harness; the library itself is C/C++/CUDA.

    lat = Lattice()
    lat.add("KQUAD", "QF", L=0.3, K1=1.2, N_KICKS=8)
    ...
    with Tracker(device=0) as trk:
        trk.load(coord)                      # (np, >=7) array, column 6 = id
        stats = trk.track(lat, n_passes=100, p_central=13700.0)
        n_left, coord_out = trk.store()

do_tracking(coord, lattice, n_passes, p_central) mirrors the reference's
do_tracking() (src/do_tracking.c:144): the beam is tracked in place,
survivors are returned first and the survivor count is returned.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtrkgpu.so")

TYPES = ["MARK", "DRIF", "EDRIFT", "KQUAD", "KSEXT", "KOCT", "CSBEND", "RFCA", "WAKE", "TRWAKE", "MAXAMP",
         "CHARGE"]
TYPE_CODE = {n: i for i, n in enumerate(TYPES)}

TRK_OK = 0


class TrackingError(RuntimeError):
    """A library call returned a negative trk_error code."""

    def __init__(self, code, message):
        super().__init__(f"trk error {code}: {message}")
        self.code = code


class _Run(ctypes.Structure):
    _fields_ = [("p_central", ctypes.c_double), ("n_passes", ctypes.c_long), ("pass_offset", ctypes.c_long),
                ("fast_math", ctypes.c_int32), ("block_size", ctypes.c_int32), ("compact_every", ctypes.c_int32),
                ("variant", ctypes.c_int32), ("time_kernels", ctypes.c_int32), ("isr_seed", ctypes.c_uint64)]


class BeamSums(ctypes.Structure):
    """trk_beam_sums: elegant's BEAM_SUMS with its BEAM_SUMS2 (index 6 = time)."""
    _fields_ = [("centroid", ctypes.c_double * 7), ("sigma", (ctypes.c_double * 7) * 7),
                ("sigman", (ctypes.c_double * 7) * 7), ("maxabs", ctypes.c_double * 7),
                ("min", ctypes.c_double * 7), ("max", ctypes.c_double * 7), ("n_part", ctypes.c_long),
                ("p0", ctypes.c_double), ("charge", ctypes.c_double)]

    @classmethod
    def zeroed(cls):
        """As zero_beam_sums leaves a BEAM_SUMS (src/compute_centroids.c:264-284)."""
        s = cls()
        for j in range(7):
            s.min[j] = 1.7976931348623157e308
            s.max[j] = -1.7976931348623157e308
        return s


SUMS_SPARSE, SUMS_NOMINMAX, SUMS_EXACT_NORMEMIT, SUMS_SECOND_ORDER = 0x1, 0x2, 0x4, 0x8


class _ApertureSearch(ctypes.Structure):
    _fields_ = [("lines", ctypes.c_int32), ("full_plane", ctypes.c_int32), ("slope_mode", ctypes.c_int32),
                ("n_splits", ctypes.c_int32), ("nx", ctypes.c_long), ("xmax", ctypes.c_double),
                ("ymax", ctypes.c_double), ("xpmax", ctypes.c_double), ("ypmax", ctypes.c_double),
                ("split_fraction", ctypes.c_double), ("orbit", ctypes.c_double * 6)]


class _ApertureGrid(ctypes.Structure):
    _fields_ = [("delta_mode", ctypes.c_int32), ("reserved", ctypes.c_int32), ("nx", ctypes.c_long),
                ("ny", ctypes.c_long), ("ndelta", ctypes.c_long), ("xmin", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymin", ctypes.c_double), ("ymax", ctypes.c_double), ("deltamin", ctypes.c_double),
                ("deltamax", ctypes.c_double), ("orbit", ctypes.c_double * 6)]


class _Stats(ctypes.Structure):
    _fields_ = [("n_total", ctypes.c_long), ("n_left", ctypes.c_long), ("particle_passes", ctypes.c_long),
                ("device_ms", ctypes.c_double), ("kernel_launches", ctypes.c_long), ("p_central", ctypes.c_double),
                ("track_ms", ctypes.c_double), ("track_launches", ctypes.c_long)]


_lib = None


_SUM_F64 = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t)
_SUM_U64 = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t)
_SUM_I64 = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_size_t)
_GATHER_F64 = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.c_size_t)


class _Exchange(ctypes.Structure):
    """trk_exchange: the caller's host-side collectives (include/trk.h)."""
    _fields_ = [("user", ctypes.c_void_p), ("sum_f64", _SUM_F64), ("sum_u64", _SUM_U64), ("sum_i64", _SUM_I64),
                ("gather_f64", _GATHER_F64)]


def _declare(lib):
    P = ctypes.c_void_p
    D = ctypes.c_double
    L = ctypes.c_long
    I = ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    sig = {
        "trk_last_error": (ctypes.c_char_p, []),
        "trk_comm_get_unique_id": (I, [P]),
        "trk_ensemble_variant": (I, [P]),
        "trk_context_set_comm": (I, [P, P, I, I]),
        "trk_context_set_exchange": (I, [P, P, I, I]),
        "trk_context_comm": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "trk_abi_version": (I, []),
        "trk_test_fail_allocation": (I, [I]),
        "trk_type_code": (I, [ctypes.c_char_p]),
        "trk_param_count": (I, [I]),
        "trk_param_name": (ctypes.c_char_p, [I, I]),
        "trk_param_default": (D, [I, I]),
        "trk_param_index": (I, [I, ctypes.c_char_p]),
        "trk_lattice_create": (I, [ctypes.POINTER(P)]),
        "trk_lattice_destroy": (None, [P]),
        "trk_lattice_add": (I, [P, I, ctypes.c_char_p, ctypes.POINTER(I)]),
        "trk_lattice_set": (I, [P, I, ctypes.c_char_p, D]),
        "trk_lattice_get": (I, [P, I, ctypes.c_char_p, DP]),
        "trk_lattice_length": (I, [P]),
        "trk_lattice_set_wake": (I, [P, I, DP, DP, DP, L]),
        "trk_lattice_parse": (I, [P, ctypes.c_char_p, ctypes.c_char_p]),
        "trk_lattice_total_length": (D, [P]),
        "trk_run_defaults": (None, [ctypes.POINTER(_Run)]),
        "trk_context_create": (I, [ctypes.POINTER(P), I]),
        "trk_context_destroy": (None, [P]),
        "trk_context_stream": (P, [P]),
        "trk_beam_load": (I, [P, DP, L, L]),
        "trk_beam_load_device": (I, [P, P, L, L]),
        "trk_beam_store": (I, [P, DP, L, ctypes.POINTER(L), ctypes.POINTER(L), ctypes.POINTER(ctypes.c_int32)]),
        "trk_beam_count": (I, [P, ctypes.POINTER(L)]),
        "trk_beam_device_columns": (I, [P, ctypes.POINTER(P), ctypes.POINTER(L), ctypes.POINTER(P)]),
        "trk_track": (I, [P, P, ctypes.POINTER(_Run), ctypes.POINTER(_Stats)]),
        "trk_track_ensemble": (I, [P, ctypes.POINTER(P), I, ctypes.POINTER(L), ctypes.POINTER(_Run),
                                   ctypes.POINTER(_Stats)]),
        "trk_adjoint": (I, [P, P, ctypes.POINTER(_Run), D, DP, DP, I]),
        "trk_beam_centroids": (I, [P, DP, ctypes.POINTER(L)]),
        "trk_accumulate_beam_sums": (I, [P, ctypes.POINTER(BeamSums), D, D, DP, D, D, L, L, ctypes.c_uint]),
        "trk_match_energy": (I, [P, DP, I]),
        "trk_sort_by_id": (I, [P]),
        "trk_aperture_search_lines": (I, [P, ctypes.POINTER(P), I, ctypes.POINTER(_ApertureSearch),
                                          ctypes.POINTER(_Run), DP, DP, DP, DP, DP, DP, DP, DP]),
        "trk_aperture_search_grid": (I, [P, ctypes.POINTER(P), I, ctypes.POINTER(_ApertureGrid),
                                         ctypes.POINTER(_Run), DP, DP, DP, DP, DP, DP, DP]),
        "trk_adjoint_ensemble": (I, [P, ctypes.POINTER(P), I, ctypes.POINTER(L), ctypes.POINTER(_Run), D, DP, DP, I]),
        "trk_adjoint_param_count": (I, [P]),
        "trk_objective": (I, [P, D, DP]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args


def load_library(path=None):
    """Load libtrkgpu.so; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is not built; run elegant_b200/build.py (or __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    _declare(lib)
    if path is None:
        _lib = lib
    return lib


def _check(lib, rc):
    if rc < 0:
        raise TrackingError(rc, lib.trk_last_error().decode(errors="replace"))
    return rc


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Lattice:
    """An ordered element list with the reference's parameter names.

    Kept in Python so the same lattice can be instantiated in the product
    library and in the CPU oracle (both expose the trk_lattice_* C API)."""

    def __init__(self):
        self.elements = []  # (type, name, {param: value}, wake tuple or None)

    def add(self, type_name, name=None, **params):
        t = type_name.upper()
        if t not in TYPE_CODE:
            raise ValueError(f"element type {type_name} is not on this path")
        self.elements.append([t, name or t, dict((k.upper(), float(v)) for k, v in params.items()), None])
        return len(self.elements) - 1

    def set(self, index, param, value):
        self.elements[index][2][param.upper()] = float(value)

    def set_wake(self, index, t, W, Wy=None):
        self.elements[index][3] = (np.ascontiguousarray(t, dtype=np.float64),
                                   np.ascontiguousarray(W, dtype=np.float64),
                                   None if Wy is None else np.ascontiguousarray(Wy, dtype=np.float64))

    def extend(self, other, times=1):
        for _ in range(times):
            for e in other.elements:
                self.elements.append([e[0], e[1], dict(e[2]), e[3]])
        return self

    def __len__(self):
        return len(self.elements)

    def indices(self, type_name):
        return [i for i, e in enumerate(self.elements) if e[0] == type_name.upper()]

    def native(self, lib):
        """Build a trk_lattice in `lib` (library or oracle); returns a handle."""
        return _NativeLattice(lib, self)

    def total_length(self):
        tot = 0.0
        for t, _, p, _ in self.elements:
            if t in ("DRIF", "EDRIFT", "KQUAD", "KSEXT", "KOCT", "CSBEND", "RFCA"):
                tot += p.get("L", 0.0)
        return tot


class _NativeLattice:
    def __init__(self, lib, lat):
        self.lib = lib
        self.ptr = ctypes.c_void_p()
        _check(lib, lib.trk_lattice_create(ctypes.byref(self.ptr)))
        self._keep = []
        try:
            for t, name, params, wake in lat.elements:
                idx = ctypes.c_int()
                _check(lib, lib.trk_lattice_add(self.ptr, TYPE_CODE[t], name.encode(), ctypes.byref(idx)))
                for k, v in params.items():
                    _check(lib, lib.trk_lattice_set(self.ptr, idx.value, k.encode(), v))
                if wake is not None:
                    tt, W, Wy = wake
                    _check(lib, lib.trk_lattice_set_wake(self.ptr, idx.value, _dptr(tt), _dptr(W),
                                                         _dptr(Wy) if Wy is not None else None, len(tt)))
        except Exception:
            lib.trk_lattice_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()  # destroyed: close() and __del__ must not free it again
            raise

    def close(self):
        if self.ptr:
            self.lib.trk_lattice_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Stats(dict):
    pass


class Tracker:
    """A device context (one CUDA stream on one GPU) holding a resident beam."""

    def __init__(self, device=0, lib=None):
        self.lib = lib or load_library()
        self.ctx = ctypes.c_void_p()
        _check(self.lib, self.lib.trk_context_create(ctypes.byref(self.ctx), device))
        self._lat_cache = {}

    def close(self):
        if self.ctx:
            self.lib.trk_context_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, coord):
        a = np.ascontiguousarray(coord, dtype=np.float64)
        if a.ndim != 2 or a.shape[1] < 7:
            raise ValueError("beam must be (np, >=7)")
        self.np = a.shape[0]
        _check(self.lib, self.lib.trk_beam_load(self.ctx, _dptr(a), a.shape[0], a.shape[1]))

    def load_device(self, ptr, np_, ld):
        self.np = np_
        _check(self.lib, self.lib.trk_beam_load_device(self.ctx, ctypes.c_void_p(ptr), np_, ld))

    def store(self, stride=7, with_loss=False, out=None):
        """Beam rows back to the host (survivors first).  `out`, if given, is
        a C-contiguous float64 (np, stride) array to fill (e.g. pinned
        memory); otherwise a new array is returned."""
        if out is None:
            out = np.zeros((self.np, stride), dtype=np.float64)
        elif out.shape != (self.np, stride) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (np, stride)")
        n_left = ctypes.c_long()
        if with_loss:
            lp = np.empty(self.np, dtype=np.int64)
            le = np.empty(self.np, dtype=np.int32)
            _check(self.lib, self.lib.trk_beam_store(
                self.ctx, _dptr(out), stride, ctypes.byref(n_left),
                lp.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), le.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
            return n_left.value, out, lp, le
        _check(self.lib, self.lib.trk_beam_store(self.ctx, _dptr(out), stride, ctypes.byref(n_left), None, None))
        return n_left.value, out

    def track_ensemble(self, lattices, counts, n_passes, p_central, pass_offset=0, fast=True, variant=-1,
                       compact_every=None):
        """Track the loaded beam as len(lattices) variants: variant v owns the
        next counts[v] particles (in load order).  The lattices must share
        one element structure.  compact_every: passes between survivor
        compactions (0 = never; None = the library default, 64).  Returns the
        run statistics plus the launch shape used ("variant")."""
        nats = [self.native(lat) for lat in lattices]
        arr = (ctypes.c_void_p * len(nats))(*[n.ptr.value for n in nats])
        offs = np.concatenate([[0], np.cumsum(np.asarray(counts, dtype=np.int64))]).astype(np.int64)
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = p_central
        run.n_passes = n_passes
        run.pass_offset = pass_offset
        run.fast_math = 1 if fast else 0
        run.variant = variant
        if compact_every is not None:
            run.compact_every = compact_every
        st = _Stats()
        _check(self.lib, self.lib.trk_track_ensemble(
            self.ctx, arr, len(nats),
            offs.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), ctypes.byref(run), ctypes.byref(st)))
        out = _stats_dict(st)
        out["variant"] = self.lib.trk_ensemble_variant(self.ctx)
        return out

    def adjoint(self, lattice, n_passes, p_central, centroid_weight=0.0, pass_offset=0, with_grad=True):
        """Track the loaded beam n_passes passes and return (loss, gradient):
        loss = mean(x^2 + y^2) + w (mean(x)^2 + mean(y)^2) over survivors,
        gradient with respect to every KQUAD K1 and KSEXT K2 in lattice order
        (reverse-mode adjoint on the device).  The beam is left at its final
        state."""
        nat = self.native(lattice)
        n = _check(self.lib, self.lib.trk_adjoint_param_count(nat.ptr))
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = p_central
        run.n_passes = n_passes
        run.pass_offset = pass_offset
        loss = ctypes.c_double()
        g = np.zeros(max(n, 1))
        _check(self.lib, self.lib.trk_adjoint(self.ctx, nat.ptr, ctypes.byref(run), centroid_weight, ctypes.byref(loss),
                                              _dptr(g) if with_grad else None, n))
        return loss.value, g[:n]

    def adjoint_ensemble(self, lattices, counts, n_passes, p_central, centroid_weight=0.0, pass_offset=0,
                         with_grad=True):
        """The batched adjoint: the loaded beam tracked as len(lattices)
        variants (variant v owns the next counts[v] particles) and, per
        variant, (loss over its survivors, gradient with respect to its KQUAD
        K1 and KSEXT K2 values).  Returns (losses[V], gradients[V, P])."""
        nats = [self.native(lat) for lat in lattices]
        arr = (ctypes.c_void_p * len(nats))(*[n.ptr.value for n in nats])
        offs = np.concatenate([[0], np.cumsum(np.asarray(counts, dtype=np.int64))]).astype(np.int64)
        n = _check(self.lib, self.lib.trk_adjoint_param_count(nats[0].ptr))
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = p_central
        run.n_passes = n_passes
        run.pass_offset = pass_offset
        V = len(nats)
        loss = np.zeros(V)
        g = np.zeros(max(n * V, 1))
        _check(self.lib, self.lib.trk_adjoint_ensemble(
            self.ctx, arr, V, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), ctypes.byref(run),
            centroid_weight, _dptr(loss), _dptr(g) if with_grad else None, n * V))
        return loss, g[:n * V].reshape(V, n)

    def centroids(self):
        """compute_centroids of the surviving particles: (centroid[6], count)."""
        c = np.zeros(6)
        n = ctypes.c_long()
        _check(self.lib, self.lib.trk_beam_centroids(self.ctx, _dptr(c), ctypes.byref(n)))
        return c, n.value

    def accumulate_beam_sums(self, sums, p_central, mp_charge=0.0, time=None, t_min=0.0, t_max=0.0, start_pid=-1,
                             end_pid=-1, flags=SUMS_SECOND_ORDER):
        """accumulate_beam_sums of the surviving particles into `sums` (BeamSums)."""
        tv = None if time is None else np.ascontiguousarray(time, dtype=np.float64)
        _check(self.lib, self.lib.trk_accumulate_beam_sums(self.ctx, ctypes.byref(sums), p_central, mp_charge,
                                                           None if tv is None else _dptr(tv), t_min, t_max,
                                                           start_pid, end_pid, flags))
        return sums

    def match_energy(self, p_central, change_beam=0):
        """do_match_energy on the device beam; returns the (new) central momentum."""
        pc = ctypes.c_double(p_central)
        _check(self.lib, self.lib.trk_match_energy(self.ctx, ctypes.byref(pc), int(change_beam)))
        return pc.value

    def aperture_search_lines(self, lattices, p_central, n_passes, lines, nx, xmax, ymax, n_splits=0,
                              split_fraction=0.5, full_plane=0, slope_mode=0, xpmax=0.0, ypmax=0.0, orbit=None,
                              fast=True, variant=-1):
        """elegant's line-mode aperture search for one lattice or a list of
        error-seed lattices, every point of a sweep in one launch.  Returns a
        dict of (variants, lines) arrays x_limit, y_limit, x_clipped,
        y_clipped, x_lost, y_lost, s_lost and area (variants,).  The loaded
        beam is replaced."""
        lats = lattices if isinstance(lattices, (list, tuple)) else [lattices]
        nats = [self.native(lat) for lat in lats]
        arr = (ctypes.c_void_p * len(nats))(*[n.ptr.value for n in nats])
        S = _ApertureSearch()
        S.lines, S.full_plane, S.slope_mode, S.n_splits = lines, full_plane, slope_mode, n_splits
        S.nx, S.xmax, S.ymax, S.xpmax, S.ypmax = nx, xmax, ymax, xpmax, ypmax
        S.split_fraction = split_fraction
        for k, v in enumerate(np.zeros(6) if orbit is None else orbit):
            S.orbit[k] = float(v)
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = p_central
        run.n_passes = n_passes
        run.fast_math = 1 if fast else 0
        run.variant = variant
        V = len(nats)
        out = {k: np.zeros(V * lines) for k in ("x_limit", "y_limit", "x_clipped", "y_clipped", "x_lost", "y_lost",
                                                 "s_lost")}
        area = np.zeros(V)
        _check(self.lib, self.lib.trk_aperture_search_lines(
            self.ctx, arr, V, ctypes.byref(S), ctypes.byref(run), _dptr(out["x_limit"]), _dptr(out["y_limit"]),
            _dptr(out["x_clipped"]), _dptr(out["y_clipped"]), _dptr(out["x_lost"]), _dptr(out["y_lost"]),
            _dptr(out["s_lost"]), _dptr(area)))
        res = {k: v.reshape(V, lines) for k, v in out.items()}
        res["area"] = area
        return res

    def aperture_search_grid(self, lattices, p_central, n_passes, nx=0, ny=0, xmin=0.0, xmax=0.0, ymin=0.0, ymax=0.0,
                             delta_mode=0, ndelta=0, deltamin=0.0, deltamax=0.0, orbit=None, fast=True, variant=-1):
        """elegant's grid-mode aperture search for one lattice or a list of
        error-seed lattices.  Returns a dict of (variants, 2, nu) arrays
        u_limit, v_limit, x_lost, y_lost, s_lost, delta_lost (side 1 only
        when the v range reaches below zero) and area (variants,).  The
        loaded beam is replaced."""
        lats = lattices if isinstance(lattices, (list, tuple)) else [lattices]
        nats = [self.native(lat) for lat in lats]
        arr = (ctypes.c_void_p * len(nats))(*[n.ptr.value for n in nats])
        G = _ApertureGrid()
        G.delta_mode, G.nx, G.ny, G.ndelta = delta_mode, nx, ny, ndelta
        G.xmin, G.xmax, G.ymin, G.ymax, G.deltamin, G.deltamax = xmin, xmax, ymin, ymax, deltamin, deltamax
        for k, v in enumerate(np.zeros(6) if orbit is None else orbit):
            G.orbit[k] = float(v)
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        run.p_central = p_central
        run.n_passes = n_passes
        run.fast_math = 1 if fast else 0
        run.variant = variant
        V = len(nats)
        nu = ndelta if delta_mode else nx
        out = {k: np.zeros(V * 2 * max(nu, 1)) for k in ("u_limit", "v_limit", "x_lost", "y_lost", "s_lost",
                                                          "delta_lost")}
        area = np.zeros(V)
        _check(self.lib, self.lib.trk_aperture_search_grid(
            self.ctx, arr, V, ctypes.byref(G), ctypes.byref(run), _dptr(out["u_limit"]), _dptr(out["v_limit"]),
            _dptr(out["x_lost"]), _dptr(out["y_lost"]), _dptr(out["s_lost"]), _dptr(out["delta_lost"]),
            _dptr(area)))
        res = {k: v.reshape(V, 2, -1) for k, v in out.items()}
        res["area"] = area
        return res

    def sort_by_id(self):
        """Survivors in increasing particle ID (lost particles after them)."""
        _check(self.lib, self.lib.trk_sort_by_id(self.ctx))

    def objective(self, centroid_weight=0.0):
        """The adjoint's loss function on the device beam as it is."""
        v = ctypes.c_double()
        _check(self.lib, self.lib.trk_objective(self.ctx, centroid_weight, ctypes.byref(v)))
        return v.value

    def set_comm(self, unique_id, nranks, rank):
        """Join a sharded run: `unique_id` (128 bytes from nccl_unique_id() on
        one rank) shared by all ranks; nranks <= 0 leaves it."""
        buf = ctypes.create_string_buffer(bytes(unique_id), 128)
        _check(self.lib, self.lib.trk_context_set_comm(self.ctx, buf, nranks, rank))

    def set_exchange(self, sum_f64, sum_u64, sum_i64, gather_f64, nranks, rank):
        """Join a sharded run whose collectives the caller performs on host
        arrays (an MPI or gloo host): sum_f64/sum_u64/sum_i64(a) sum the
        numpy array `a` element-wise over the ranks in place;
        gather_f64(send, recv) fills recv (nranks * len(send)) with every
        rank's send in rank order.  nranks <= 0 leaves the run."""
        def wrap_sum(fn, dtype):
            def cb(_user, buf, n):
                try:
                    fn(np.ctypeslib.as_array(buf, shape=(n,)) if n else np.zeros(0, dtype))
                    return 0
                except Exception:  # the library reports the failure as TRK_ERR_NCCL
                    return 1
            return cb

        def cb_gather(_user, send, recv, n):
            try:
                gather_f64(np.ctypeslib.as_array(send, shape=(n,)), np.ctypeslib.as_array(recv, shape=(n * nranks,)))
                return 0
            except Exception:
                return 1

        ex = _Exchange(None, _SUM_F64(wrap_sum(sum_f64, np.float64)), _SUM_U64(wrap_sum(sum_u64, np.uint64)),
                       _SUM_I64(wrap_sum(sum_i64, np.int64)), _GATHER_F64(cb_gather))
        self._exchange = ex  # the library holds the pointer while the exchange is set
        _check(self.lib, self.lib.trk_context_set_exchange(self.ctx, ctypes.byref(ex), nranks, rank))

    def count(self):
        n = ctypes.c_long()
        _check(self.lib, self.lib.trk_beam_count(self.ctx, ctypes.byref(n)))
        return n.value

    def columns(self):
        cols = (ctypes.c_void_p * 7)()
        n = ctypes.c_long()
        loss = (ctypes.c_void_p * 2)()
        _check(self.lib, self.lib.trk_beam_device_columns(self.ctx, cols, ctypes.byref(n), loss))
        return [c for c in cols], n.value, [l for l in loss]

    def stream(self):
        return self.lib.trk_context_stream(self.ctx)

    def native(self, lattice):
        key = id(lattice)
        nat = self._lat_cache.get(key)
        if nat is None or nat[0] is not lattice or nat[2] != _lattice_signature(lattice):
            nat = (lattice, lattice.native(self.lib), _lattice_signature(lattice))
            self._lat_cache[key] = nat
        return nat[1]

    def track(self, lattice, n_passes, p_central, pass_offset=0, fast=True, variant=-1, time_kernels=False,
              isr_seed=0, compact_every=None):
        """Track the loaded beam n_passes passes (trk_track).  compact_every:
        passes between survivor compactions in fused multi-pass runs (0 =
        never; None = the library default, 64)."""
        nat = self.native(lattice)
        run = _Run()
        self.lib.trk_run_defaults(ctypes.byref(run))
        if compact_every is not None:
            run.compact_every = compact_every
        run.p_central = p_central
        run.n_passes = n_passes
        run.pass_offset = pass_offset
        run.fast_math = 1 if fast else 0
        run.variant = variant
        run.isr_seed = isr_seed
        run.time_kernels = 1 if time_kernels else 0
        st = _Stats()
        _check(self.lib, self.lib.trk_track(self.ctx, nat.ptr, ctypes.byref(run), ctypes.byref(st)))
        return Stats(n_total=st.n_total, n_left=st.n_left, particle_passes=st.particle_passes,
                     device_ms=st.device_ms, kernel_launches=st.kernel_launches, p_central=st.p_central,
                     track_ms=st.track_ms, track_launches=st.track_launches)


def _stats_dict(st):
    return Stats(n_total=st.n_total, n_left=st.n_left, particle_passes=st.particle_passes,
                 device_ms=st.device_ms, kernel_launches=st.kernel_launches, p_central=st.p_central,
                 track_ms=st.track_ms, track_launches=st.track_launches)


def nccl_unique_id():
    """128-byte NCCL id for Tracker.set_comm (call on one rank, share it)."""
    lib = load_library()
    buf = ctypes.create_string_buffer(128)
    _check(lib, lib.trk_comm_get_unique_id(buf))
    return buf.raw


def _lattice_signature(lat):
    return tuple((t, n, tuple(sorted(p.items())), None if w is None else id(w)) for t, n, p, w in lat.elements)


def do_tracking(coord, lattice, n_passes, p_central, fast=True, device=0):
    """Track `coord` (np x >=7, modified in place: survivors first, then lost
    particles) through n_passes of `lattice`; returns the survivor count, as
    the reference's do_tracking() (src/do_tracking.c:144)."""
    with Tracker(device) as trk:
        trk.load(coord)
        trk.track(lattice, n_passes, p_central, fast=fast)
        n_left, out = trk.store(stride=coord.shape[1])
    coord[:, :] = out
    return n_left
