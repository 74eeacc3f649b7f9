"""trk_wake_noalloc: the WAKE kick for callers that cannot allocate device
memory where they track (their device memory belongs to their own pool
allocator, or they cannot take cudaMalloc/cudaFree's device-wide
synchronization).  Its scratch lives in a static device array, so two calls
in a row share it; each call must still match the allocating path
(trk_track on a CHARGE + WAKE lattice) exactly.

Collected last (tests/test_zz_*) so a stop-at-first-failure run has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from elegant_b200 import Lattice, Tracker, configs, load_library

pytestmark = pytest.mark.gpu

PC = configs.P_CENTRAL
CHARGE = 1e-9
MAX_BINS = 8192  # TRK_NOALLOC_MAX_BINS in include/trk.h


def _declare(lib):
    f = lib.trk_wake_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_long, ctypes.c_double, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                  ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_int, ctypes.c_void_p]
    return f


def _beam(n):
    b = configs.gaussian_beam(n, seed=31)
    b[:, 4] += 264.0  # one turn of path length, as at a WAKE after the first pass
    return b


def _reference_path(beam, t, W, fast, n_bins):
    lat = Lattice()
    lat.add("CHARGE", "Q", TOTAL=CHARGE)
    i = lat.add("WAKE", "W", N_BINS=n_bins, ALLOW_LONG_BEAM=1)
    lat.set_wake(i, t, W)
    with Tracker(0) as trk:
        trk.load(beam)
        trk.track(lat, 1, PC, fast=fast)
        n_left, out = trk.store()
    return n_left, out


@pytest.mark.parametrize("n_bins", [2000, MAX_BINS])
@pytest.mark.parametrize("fast", [True, False])
def test_wake_noalloc_matches_allocating_path(fast, n_bins):
    import torch
    lib = load_library()
    f = _declare(lib)
    n = 200_000
    beam = _beam(n)
    t, W = configs.resonator_wake(points=4096, dt=1e-12)
    dt = (t[-1] - t[0]) / (len(t) - 1)  # the spacing the allocating path derives from the table
    n_ref, ref = _reference_path(beam, t, W, fast, n_bins)
    ref = ref[np.argsort(ref[:, 6])]

    # Device memory for the caller's beam and wake table comes from two other
    # contexts (the test plays the caller that owns its memory); the entry
    # point itself allocates nothing.  The table is column 0 (x) of a
    # "beam" whose x values are W.
    with Tracker(0) as holder, Tracker(0) as table_holder:
        tb = np.zeros((len(W), 7))
        tb[:, 0] = W
        table_holder.load(tb)
        wcols, _, _ = table_holder.columns()
        for call in range(2):
            holder.load(beam)
            cols, npart, loss = holder.columns()
            assert npart == n
            colptr = (ctypes.c_void_p * 6)(*cols[:6])
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(0)[0]
            rc = f(colptr, loss[0], loss[1], n, PC, wcols[0], len(W), dt, n_bins, CHARGE / n, 1.0, 0, 1, 0,
                   1 if fast else 0, holder.stream())
            assert rc == 0, lib.trk_last_error()
            torch.cuda.synchronize()
            if call == 1:
                # the defining property: the call took no device memory
                # (the first call on a device only looks up the static
                # array's address, which allocates nothing either)
                assert torch.cuda.mem_get_info(0)[0] == free0
            n_left, out = holder.store()
            out = out[np.argsort(out[:, 6])]
            assert n_left == n_ref
            # same kernels on the same inputs: identical to the last bit
            assert np.array_equal(out[:, :6], ref[:, :6]), (call, np.max(np.abs(out[:, :6] - ref[:, :6])))


def test_wake_noalloc_rejects_oversized_histogram():
    lib = load_library()
    f = _declare(lib)
    colptr = (ctypes.c_void_p * 6)(*([ctypes.c_void_p(8)] * 6))
    # size checks happen on the host, before any pointer is used
    rc = f(colptr, ctypes.c_void_p(8), ctypes.c_void_p(8), 10, PC, ctypes.c_void_p(8), 100, 1e-12, 8193, 1e-12,
           1.0, 0, 1, 0, 1, None)
    assert rc == -1
    assert b"n_bins" in lib.trk_last_error()
