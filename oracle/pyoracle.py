"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle (liboracle.so).

The oracle restates elegant's element functions and do_tracking loop in C
(oracle/trk_oracle.c).  Tests, smoke() and bench.py's CPU baseline call it as
the checker; the product library never does.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
STRIDE = 9


class _Result(ctypes.Structure):
    _fields_ = [("n_left", ctypes.c_long), ("particle_passes", ctypes.c_long), ("p_central", ctypes.c_double)]


_lib = None


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    P, D, L, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_long, ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    lib.trk_last_error.restype = ctypes.c_char_p
    lib.trk_lattice_create.argtypes = [ctypes.POINTER(P)]
    lib.trk_lattice_destroy.argtypes = [P]
    lib.trk_lattice_add.argtypes = [P, I, ctypes.c_char_p, ctypes.POINTER(I)]
    lib.trk_lattice_set.argtypes = [P, I, ctypes.c_char_p, D]
    lib.trk_lattice_set_wake.argtypes = [P, I, DP, DP, DP, L]
    lib.trk_lattice_parse.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
    lib.trk_lattice_length.argtypes = [P]
    lib.trk_param_index.argtypes = [I, ctypes.c_char_p]
    lib.orc_track.argtypes = [P, DP, L, L, L, DP, ctypes.POINTER(_Result)]
    lib.orc_track_element.argtypes = [P, I, DP, L, L, DP, ctypes.POINTER(L)]
    lib.orc_csbend_field_table.argtypes = [P, I, DP, DP, ctypes.POINTER(I), ctypes.POINTER(I), ctypes.POINTER(I)]
    lib.orc_set_collective.argtypes = [I, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_set_exact_sums.argtypes = [I]
    lib.orc_set_isr_seed.argtypes = [ctypes.c_ulonglong]
    lib.orc_set_cr_math.argtypes = [I]
    lib.orc_cr_selftest.argtypes = [I, D, D, I, L, ctypes.c_ulonglong, ctypes.POINTER(L), DP]
    lib.orc_cr_selftest.restype = L
    lib.orc_div_rcp_selftest.argtypes = [L, ctypes.c_ulonglong]
    lib.orc_div_rcp_selftest.restype = L
    for f in ('orc_cr_sin', 'orc_cr_cos', 'orc_cr_asin', 'orc_cr_tan'):
        getattr(lib, f).argtypes = [D]
        getattr(lib, f).restype = D
    _lib = lib
    return lib


def _check(lib, rc):
    if rc < 0:
        raise RuntimeError(f"oracle error {rc}: {lib.trk_last_error().decode(errors='replace')}")
    return rc


def set_exact_sums(on):
    load().orc_set_exact_sums(1 if on else 0)


def set_cr_math(on):
    load().orc_set_cr_math(1 if on else 0)


class modes:
    """Context manager selecting the oracle's summation and libm modes."""

    def __init__(self, exact_sums=False, cr_math=False):
        self.es, self.cr = exact_sums, cr_math

    def __enter__(self):
        set_exact_sums(self.es)
        set_cr_math(self.cr)
        return self

    def __exit__(self, *exc):
        set_exact_sums(False)
        set_cr_math(False)


_GATHER = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_long)
_SUM = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_long)
_collective_refs = None


def set_collective(world, gather=None, allsum=None):
    """Shard the oracle's collective steps over `world` ranks.  gather(send)
    returns the concatenation of every rank's send array (numpy float64);
    allsum(buf) returns the element-wise sum over ranks.  world <= 1 resets."""
    global _collective_refs
    lib = load()
    if world <= 1:
        lib.orc_set_collective(1, None, None)
        _collective_refs = None
        return

    def g(send, recv, n):
        out = gather(np.ctypeslib.as_array(send, shape=(n,)).copy())
        np.ctypeslib.as_array(recv, shape=(world * n,))[:] = out

    def sm(buf, n):
        a = np.ctypeslib.as_array(buf, shape=(n,))
        a[:] = allsum(a.copy())

    _collective_refs = (_GATHER(g), _SUM(sm))
    lib.orc_set_collective(world, ctypes.cast(_collective_refs[0], ctypes.c_void_p),
                           ctypes.cast(_collective_refs[1], ctypes.c_void_p))


def track(lattice, beam, n_passes, p_central, pass_offset=0):
    """Track an (np, >=7) beam; returns (rows (np, 9) in the reference's
    swap order, n_left, particle_passes).  Columns 7, 8 of rows hold the loss
    pass and element index (-1 for survivors)."""
    lib = load()
    nat = lattice.native(lib)
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    pc = ctypes.c_double(p_central)
    res = _Result()
    _check(lib, lib.orc_track(nat.ptr, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows.shape[0],
                              n_passes, pass_offset, ctypes.byref(pc), ctypes.byref(res)))
    nat.close()
    return rows, res.n_left, res.particle_passes


def final_p_central(lattice, beam, n_passes, p_central, pass_offset=0):
    """The central momentum after tracking (CHANGE_P0 elements move it)."""
    lib = load()
    nat = lattice.native(lib)
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    pc = ctypes.c_double(p_central)
    res = _Result()
    _check(lib, lib.orc_track(nat.ptr, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows.shape[0],
                              n_passes, pass_offset, ctypes.byref(pc), ctypes.byref(res)))
    nat.close()
    return pc.value


def track_element(lattice, element, beam, pass_index, p_central):
    lib = load()
    nat = lattice.native(lib)
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    pc = ctypes.c_double(p_central)
    n_left = ctypes.c_long()
    _check(lib, lib.orc_track_element(nat.ptr, element, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      rows.shape[0], pass_index, ctypes.byref(pc), ctypes.byref(n_left)))
    nat.close()
    return rows, n_left.value


def csbend_field_table(lattice, element):
    lib = load()
    nat = lattice.native(lib)
    Fx = np.zeros(121)
    Fy = np.zeros(121)
    eo1, hn, hs = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib, lib.orc_csbend_field_table(nat.ptr, element, Fx.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           Fy.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(eo1),
                                           ctypes.byref(hn), ctypes.byref(hs)))
    nat.close()
    return Fx.reshape(11, 11), Fy.reshape(11, 11), eo1.value, hn.value, hs.value


# ------------------------------------------------------------------------
# oracle/_ref/libref.so: elegant's own tracking sources compiled from the
# reference tree (oracle/ref/Makefile) and driven by oracle/ref/ref_driver.c.
# Present only where the reference sources were available to build it.
REF_LIB = os.path.join(HERE, "_ref", "libref.so")
_ref = None


def ref_available():
    return os.path.exists(REF_LIB)


def load_ref():
    global _ref
    if _ref is not None:
        return _ref
    if not ref_available():
        raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle/ref REF=<reference tree>)")
    lib = ctypes.CDLL(REF_LIB)
    P, D, L, I = ctypes.c_void_p, ctypes.c_double, ctypes.c_long, ctypes.c_int
    DP = ctypes.POINTER(ctypes.c_double)
    lib.trk_last_error.restype = ctypes.c_char_p
    lib.trk_lattice_create.argtypes = [ctypes.POINTER(P)]
    lib.trk_lattice_destroy.argtypes = [P]
    lib.trk_lattice_add.argtypes = [P, I, ctypes.c_char_p, ctypes.POINTER(I)]
    lib.trk_lattice_set.argtypes = [P, I, ctypes.c_char_p, D]
    lib.trk_lattice_set_wake.argtypes = [P, I, DP, DP, DP, L]
    lib.trk_lattice_length.argtypes = [P]
    lib.trk_param_count.argtypes = [I]
    lib.trk_param_name.argtypes = [I, I]
    lib.trk_param_name.restype = ctypes.c_char_p
    lib.trk_param_default.argtypes = [I, I]
    lib.trk_param_default.restype = D
    lib.ref_track.argtypes = [P, DP, L, L, L, DP, ctypes.POINTER(_Result)]
    lib.ref_do_tracking.argtypes = [P, DP, L, L, L, DP, ctypes.POINTER(_Result)]
    lib.ref_set_cr_math.argtypes = [I]
    lib.ref_set_exact_sums.argtypes = [I]
    lib.ref_param_defaults.argtypes = [I, DP, I]
    _ref = lib
    return lib


def track_ref(lattice, beam, n_passes, p_central, pass_offset=0, exact_sums=False, cr_math=False, loop="driver"):
    """As track(), through elegant's own element functions.  loop="driver":
    the element calls of do_tracking's switch in oracle/ref/ref_driver.c's
    pass loop; loop="do_tracking": elegant's own do_tracking()
    (src/do_tracking.c:144), which records no loss element (column 8 is -2
    for lost rows)."""
    lib = load_ref()
    lib.ref_set_exact_sums(1 if exact_sums else 0)
    lib.ref_set_cr_math(1 if cr_math else 0)
    nat = lattice.native(lib)
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    pc = ctypes.c_double(p_central)
    res = _Result()
    try:
        entry = lib.ref_do_tracking if loop == "do_tracking" else lib.ref_track
        _check(lib, entry(nat.ptr, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows.shape[0], n_passes,
                          pass_offset, ctypes.byref(pc), ctypes.byref(res)))
    finally:
        nat.close()
        lib.ref_set_exact_sums(0)
        lib.ref_set_cr_math(0)
    return rows, res.n_left, res.particle_passes


def ref_param_defaults(type_code):
    """The reference's default of each parameter of the lattice tables
    (NaN where the reference table lacks the name)."""
    lib = load_ref()
    out = np.zeros(128)
    n = lib.ref_param_defaults(type_code, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 128)
    if n < 0:
        raise RuntimeError("bad type")
    return out[:n]


# oracle/_ref/libref_gpu.so: the same reference sources compiled with elegant's
# HAVE_GPU hooks on, the hooks implemented over libtrkgpu.so
# (elegant_b200/hooks/trk_elegant_hooks.c); needs a GPU to run.
REF_GPU_LIB = os.path.join(HERE, "_ref", "libref_gpu.so")
_refgpu = None


def refgpu_available():
    return os.path.exists(REF_GPU_LIB)


def track_refgpu(lattice, beam, n_passes, p_central, pass_offset=0, loop="driver"):
    """As track_ref(), with every element going through elegant's GPU hooks
    into the CUDA library (parity build).  Rows come back survivors first.
    loop="do_tracking": elegant's own do_tracking() drives the hooks
    (column 8 is -2 for lost rows, as track_ref's do_tracking loop gives)."""
    global _refgpu
    if _refgpu is None:
        lib = ctypes.CDLL(REF_GPU_LIB)
        P = ctypes.c_void_p
        DP = ctypes.POINTER(ctypes.c_double)
        L, I, D = ctypes.c_long, ctypes.c_int, ctypes.c_double
        lib.trk_last_error.restype = ctypes.c_char_p
        lib.trk_lattice_create.argtypes = [ctypes.POINTER(P)]
        lib.trk_lattice_destroy.argtypes = [P]
        lib.trk_lattice_add.argtypes = [P, I, ctypes.c_char_p, ctypes.POINTER(I)]
        lib.trk_lattice_set.argtypes = [P, I, ctypes.c_char_p, D]
        lib.trk_lattice_set_wake.argtypes = [P, I, DP, DP, DP, L]
        lib.refgpu_track.argtypes = [P, DP, L, L, L, DP, ctypes.POINTER(_Result)]
        lib.refgpu_do_tracking.argtypes = [P, DP, L, L, L, DP, ctypes.POINTER(_Result)]
        _refgpu = lib
    lib = _refgpu
    nat = lattice.native(lib)
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    pc = ctypes.c_double(p_central)
    res = _Result()
    try:
        entry = lib.refgpu_do_tracking if loop == "do_tracking" else lib.refgpu_track
        _check(lib, entry(nat.ptr, rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows.shape[0], n_passes,
                          pass_offset, ctypes.byref(pc), ctypes.byref(res)))
    finally:
        nat.close()
    return rows, res.n_left, res.particle_passes


# ------------------------------------------------------------ beam observers
class BeamSums(ctypes.Structure):
    """The layout of orc_beam_sums / trk_beam_sums / elegant's BEAM_SUMS(2)."""
    _fields_ = [("centroid", ctypes.c_double * 7), ("sigma", (ctypes.c_double * 7) * 7),
                ("sigman", (ctypes.c_double * 7) * 7), ("maxabs", ctypes.c_double * 7),
                ("min", ctypes.c_double * 7), ("max", ctypes.c_double * 7), ("n_part", ctypes.c_long),
                ("p0", ctypes.c_double), ("charge", ctypes.c_double)]


def zero_beam_sums():
    """Fresh sums as zero_beam_sums leaves them (src/compute_centroids.c:264-284)."""
    s = BeamSums()
    for j in range(7):
        s.min[j] = 1.7976931348623157e308
        s.max[j] = -1.7976931348623157e308
    return s


def sums_dict(s):
    return {"centroid": np.array(s.centroid[:]), "sigma": np.array([r[:] for r in s.sigma]),
            "sigman": np.array([r[:] for r in s.sigman]), "maxabs": np.array(s.maxabs[:]),
            "min": np.array(s.min[:]), "max": np.array(s.max[:]), "n_part": s.n_part, "p0": s.p0,
            "charge": s.charge}


def _rows(beam):
    rows = np.zeros((beam.shape[0], STRIDE), dtype=np.float64)
    rows[:, :7] = beam[:, :7]
    return rows


def beam_centroids(beam):
    """compute_centroids on the rows of `beam` (all survivors)."""
    lib = load()
    lib.orc_beam_centroids.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_long, ctypes.POINTER(ctypes.c_double)]
    rows = _rows(beam)
    c = np.zeros(6)
    lib.orc_beam_centroids(rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), rows.shape[0],
                           c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return c


def accumulate_beam_sums(beam, sums, p_central, mp_charge=0.0, time=None, t_min=0.0, t_max=0.0, start_pid=-1,
                         end_pid=-1, flags=0x8):
    """accumulate_beam_sums on the rows of `beam` into `sums` (BeamSums)."""
    lib = load()
    DP = ctypes.POINTER(ctypes.c_double)
    lib.orc_accumulate_beam_sums.argtypes = [DP, ctypes.c_long, ctypes.POINTER(BeamSums), ctypes.c_double,
                                             ctypes.c_double, DP, ctypes.c_double, ctypes.c_double, ctypes.c_long,
                                             ctypes.c_long, ctypes.c_uint]
    rows = _rows(beam)
    tv = None if time is None else np.ascontiguousarray(time, dtype=np.float64)
    lib.orc_accumulate_beam_sums(rows.ctypes.data_as(DP), rows.shape[0], ctypes.byref(sums), p_central, mp_charge,
                                 None if tv is None else tv.ctypes.data_as(DP), t_min, t_max, start_pid, end_pid,
                                 flags)
    return sums


def match_energy(beam, p_central, change_beam):
    """do_match_energy on the rows of `beam`; returns (beam, p_central)."""
    lib = load()
    DP = ctypes.POINTER(ctypes.c_double)
    lib.orc_match_energy.argtypes = [DP, ctypes.c_long, DP, ctypes.c_int]
    rows = _rows(beam)
    pc = ctypes.c_double(p_central)
    lib.orc_match_energy(rows.ctypes.data_as(DP), rows.shape[0], ctypes.byref(pc), int(change_beam))
    out = beam.copy()
    out[:, :7] = rows[:, :7]
    return out, pc.value


def _observe(lib, fn, beam, p_central, mp_charge, flags, start_pid, end_pid, t_min, t_max, repeats):
    DP = ctypes.POINTER(ctypes.c_double)
    f = getattr(lib, fn)
    f.argtypes = [DP, ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_uint, ctypes.c_long, ctypes.c_long,
                  ctypes.c_double, ctypes.c_double, ctypes.c_int, DP, ctypes.POINTER(BeamSums)]
    rows = _rows(beam)
    c = np.zeros(6)
    s = BeamSums()
    _check(lib, f(rows.ctypes.data_as(DP), rows.shape[0], p_central, mp_charge, flags, start_pid, end_pid, t_min,
                  t_max, repeats, c.ctypes.data_as(DP), ctypes.byref(s)))
    return c, s


def observe_ref(beam, p_central, mp_charge=0.0, flags=0x8, start_pid=-1, end_pid=-1, t_min=0.0, t_max=0.0,
                repeats=1, exact_sums=False):
    """elegant's own compute_centroids and accumulate_beam_sums (libref.so)
    on the rows of `beam`: (centroid[6], BeamSums after `repeats`
    accumulations from zero_beam_sums)."""
    lib = load_ref()
    lib.ref_set_exact_sums(1 if exact_sums else 0)
    try:
        return _observe(lib, "ref_observe", beam, p_central, mp_charge, flags, start_pid, end_pid, t_min, t_max,
                        repeats)
    finally:
        lib.ref_set_exact_sums(0)


def observe_refgpu(beam, p_central, mp_charge=0.0, flags=0x8, start_pid=-1, end_pid=-1, t_min=0.0, t_max=0.0,
                   repeats=1):
    """As observe_ref(), with the calls going through elegant's GPU hooks
    into the CUDA library (libref_gpu.so)."""
    lib = ctypes.CDLL(REF_GPU_LIB)
    lib.trk_last_error.restype = ctypes.c_char_p
    return _observe(lib, "refgpu_observe", beam, p_central, mp_charge, flags, start_pid, end_pid, t_min, t_max,
                    repeats)


# ------------------------------------------------------------ aperture search
def aperture_search_grid(lattice, p_central, n_passes, nx=0, ny=0, xmin=0.0, xmax=0.0, ymin=0.0, ymax=0.0,
                         delta_mode=0, ndelta=0, deltamin=0.0, deltamax=0.0, orbit=None):
    """do_aperture_search_grid (src/aperture_search.c:1236-1521) restated:
    each side's grid tracked by the oracle as one beam (IDs 1.. in grid
    order), then the reference's reduction over the survivor rows and the
    lost rows in their order.  Returns dict of (2, nu) arrays u_limit,
    v_limit, x_lost, y_lost, s_lost, delta_lost and the area."""
    orbit = np.zeros(6) if orbit is None else np.asarray(orbit, dtype=np.float64)
    if delta_mode == 1:
        icu, icv, nu, umin, umax, nv, vmin, vmax = 5, 0, ndelta, deltamin, deltamax, nx, xmin, xmax
    elif delta_mode == 2:
        icu, icv, nu, umin, umax, nv, vmin, vmax = 5, 2, ndelta, deltamin, deltamax, ny, ymin, ymax
    else:
        icu, icv, nu, umin, umax, nv, vmin, vmax = 0, 2, nx, xmin, xmax, ny, ymin, ymax
    big = 1.7976931348623157e308
    du = (umax - umin) / (nu - 1)
    out = {k: np.zeros((2, nu)) for k in ("u_limit", "v_limit")}
    out.update({k: np.full((2, nu), big) for k in ("x_lost", "y_lost", "s_lost", "delta_lost")})
    area = 0.0
    for side in range(2 if vmin < 0 else 1):
        dv = vmax / (nv - 1) if side == 0 else vmin / (nv - 1)
        b = np.zeros((nu * nv, 7))
        ip = 0
        for iu in range(nu):
            for iv in range(nv):
                b[ip, icu] = iu * du + umin
                b[ip, icv] = iv * dv
                b[ip, 6] = ip + 1
                ip += 1
        b[:, :6] += orbit
        rows, n_left, _ = track(lattice, b, n_passes, p_central)
        vl = [0.0] * nu
        vl1 = [(vmax if side == 0 else vmin) + dv] * nu
        for ip in range(n_left):
            pid = int(rows[ip, 6])
            iu, iv = (pid - 1) // nv, (pid - 1) % nv
            v = iv * dv
            if (side == 0 and v > vl[iu]) or (side == 1 and v < vl[iu]):
                vl[iu] = v
        for ip in range(n_left, nu * nv):
            pid = int(rows[ip, 6])
            iu, iv = (pid - 1) // nv, (pid - 1) % nv
            v = iv * dv
            if (side == 0 and v < vl[iu]) or (side == 1 and v > vl[iu]):
                vl[iu] = v
            if (side == 0 and v < vl1[iu]) or (side == 1 and v > vl1[iu]):
                vl1[iu] = v
                out["x_lost"][side, iu] = rows[ip, 0]
                out["y_lost"][side, iu] = rows[ip, 2]
                out["s_lost"][side, iu] = rows[ip, 4]
                out["delta_lost"][side, iu] = rows[ip, 5]
        if n_left:
            for iu in range(nu):
                area += abs(vl[iu] * du)
        for iu in range(nu):
            out["u_limit"][side, iu] = iu * du + umin
            out["v_limit"][side, iu] = vl[iu]
    out["area"] = area
    return out


def aperture_search_lines(lattice, p_central, n_passes, lines, nx, xmax, ymax, n_splits=0, split_fraction=0.5,
                          full_plane=0, slope_mode=0, xpmax=0.0, ypmax=0.0, orbit=None, area_fn=None):
    """do_aperture_search_line (src/aperture_search.c:985-1234) restated
    serially: one particle at a time along each line, each sweep stopping at
    the first loss, tracked by the oracle.  Returns dict with x_limit,
    y_limit, x_lost, y_lost, s_lost per line, origin_stable, and, if
    area_fn is given (the trimming routine), the clipped limits and area."""
    import math
    orbit = np.zeros(6) if orbit is None else np.asarray(orbit, dtype=np.float64)
    if lines == 1:
        dxf, dyf = [1.0], [1.0]
    elif lines == 2:
        dxf, dyf = [-1.0, 1.0], [1.0, 1.0]
    elif lines == 3:
        dxf, dyf = [0.0, 1 / math.sqrt(2), 1.0], [1.0, 1 / math.sqrt(2), 0.0]
    else:
        dtheta = (math.pi if full_plane == 0 else 2 * math.pi) / (lines - 1)
        dxf = [math.sin(-math.pi / 2 + dtheta * k) for k in range(lines)]
        dyf = [math.cos(-math.pi / 2 + dtheta * k) for k in range(lines)]
        dxf = [0.0 if abs(v) < 1e-6 else v for v in dxf]
        dyf = [0.0 if abs(v) < 1e-6 else v for v in dyf]
    big = 1.7976931348623157e308
    origin_stable = False
    xlim, ylim, xl_, yl_, sl_ = [], [], [], [], []
    for line in range(lines):
        if dxf[line] > 0:
            xs = ys = -1.0
        else:
            ys = -1.0
            xs = 1.0
        xl = yl = sl = big
        for split in range(n_splits + 1):
            if split == 0:
                ex, ey = (xpmax, ypmax) if slope_mode else (xmax, ymax)
                dx = ex / (nx - 1) * dxf[line]
                dy = ey / (nx - 1) * dyf[line]
                x0 = y0 = 0.0
                steps = nx
            else:
                x0, y0 = xs, ys
                dx *= split_fraction
                dy *= split_fraction
                x0 += dx
                y0 += dy
                steps = max(1, int(1 / split_fraction - 0.5))
            for index in range(steps):
                if index != 0 or split != 0 or not origin_stable:
                    b = np.zeros((1, 7))
                    b[0, :6] = orbit
                    if not slope_mode:
                        b[0, 0] = index * dx + x0 + orbit[0]
                        b[0, 2] = index * dy + y0 + orbit[2]
                    else:
                        b[0, 1] = index * dx + x0 + orbit[1]
                        b[0, 3] = index * dy + y0 + orbit[3]
                    b[0, 6] = 1
                    rows, n_left, _ = track(lattice, b, n_passes, p_central)
                    if n_left != 1:
                        xl, yl, sl = rows[0, 0], rows[0, 2], rows[0, 4]
                        break
                if index == 0 and split == 0:
                    origin_stable = True
                xk, yk = x0 + index * dx, y0 + index * dy
                if dxf[line]:
                    if (dxf[line] > 0 and xs < xk) or (dxf[line] < 0 and xs > xk):
                        xs, ys = xk, yk
                elif ys < yk:
                    xs, ys = xk, yk
        xlim.append(xs)
        ylim.append(ys)
        xl_.append(xl)
        yl_.append(yl)
        sl_.append(sl)
    out = {"x_limit": np.array(xlim), "y_limit": np.array(ylim), "x_lost": np.array(xl_), "y_lost": np.array(yl_),
           "s_lost": np.array(sl_), "origin_stable": origin_stable, "dxf": np.array(dxf), "dyf": np.array(dyf)}
    if area_fn is not None:
        xc, yc = out["x_limit"].copy(), out["y_limit"].copy()
        out["area"] = area_fn(xc, yc, out["dxf"], out["dyf"], full_plane) if origin_stable and lines > 1 else 0.0
        out["x_clipped"], out["y_clipped"] = xc, yc
    return out


def trim_aperture_ref(x, y, dxf, dyf, full_plane):
    """elegant's own trimApertureSearchResult (libref.so), clipping x, y in place."""
    lib = load_ref()
    DP = ctypes.POINTER(ctypes.c_double)
    lib.trimApertureSearchResult.argtypes = [ctypes.c_long, DP, DP, DP, DP, ctypes.c_long]
    lib.trimApertureSearchResult.restype = ctypes.c_double
    dxf = np.ascontiguousarray(dxf, dtype=np.float64)
    dyf = np.ascontiguousarray(dyf, dtype=np.float64)
    return lib.trimApertureSearchResult(len(x), x.ctypes.data_as(DP), y.ctypes.data_as(DP), dxf.ctypes.data_as(DP),
                                        dyf.ctypes.data_as(DP), int(full_plane))


def set_isr_seed(seed):
    """Seed of the oracle's incoherent-radiation deviates (as trk_run.isr_seed)."""
    load().orc_set_isr_seed(int(seed))
