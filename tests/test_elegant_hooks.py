"""The drop-in as an elegant build uses it: elegant's own tracking sources
compiled with -DHAVE_GPU (oracle/_ref/libref_gpu.so), whose element functions
call the GPU hooks of elegant_b200/hooks/trk_elegant_hooks.c, which run the
elements in libtrkgpu.so (parity build).  Against the same sources compiled
without the hooks (CPU, correctly rounded libm, double-double sums): every
coordinate, survivor, loss pass and loss element bit for bit.  The pass loop
is either the reference driver's (oracle/ref/ref_driver.c) or elegant's own
do_tracking() (src/do_tracking.c), which then calls gpuBaseInit,
setElementGpuData and gpuBaseDealloc itself, as an elegant GPU build does.
"""
import math

import numpy as np
import pytest

from elegant_b200 import Lattice, configs
from oracle import pyoracle
from tests.cases import ELEMENT_CASES

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (pyoracle.refgpu_available() and pyoracle.ref_available()),
                                 reason="oracle/_ref/libref_gpu.so not built")]
PC = configs.P_CENTRAL


def _same(lat, beam, passes):
    g, gn, ge = pyoracle.track_refgpu(lat, beam, passes, PC)
    c, cn, ce = pyoracle.track_ref(lat, beam, passes, PC, exact_sums=True, cr_math=True)
    assert gn == cn
    a = g[np.argsort(g[:, 6])]
    b = c[np.argsort(c[:, 6])]
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{(~same).any(axis=1).sum()} rows differ; columns {(~same).sum(axis=0)}"


@pytest.mark.parametrize("name", sorted(ELEMENT_CASES))
def test_element_through_hooks(name):
    _same(ELEMENT_CASES[name], configs.gaussian_beam(2000, seed=71), 2)


def test_rf_wake_ring_through_hooks():
    _same(configs.c2_lattice(cells=4, n_bins=2000), configs.gaussian_beam(3000, seed=72), 3)


def test_lossy_ring_through_hooks():
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.004, Y_MAX=0.003)
    lat.extend(configs.c1_lattice(cells=2))
    lat.add("MAXAMP", "AP2", X_MAX=0.005, Y_MAX=0.004, ELLIPTICAL=1)
    lat.extend(configs.c1_lattice(cells=2))
    beam = configs.gaussian_beam(3000, seed=73, sigma_x=2e-3, sigma_xp=2e-4)
    beam[5, 0] = np.nan
    beam[9, 1] = 2.0
    _same(lat, beam, 3)


def _same_do_tracking(lat, beam, passes, pass_offset=0):
    g, gn, ge = pyoracle.track_refgpu(lat, beam, passes, PC, pass_offset=pass_offset, loop="do_tracking")
    c, cn, ce = pyoracle.track_ref(lat, beam, passes, PC, pass_offset=pass_offset, exact_sums=True, cr_math=True,
                                   loop="do_tracking")
    assert gn == cn and ge == ce, (gn, cn, ge, ce)
    a = g[np.argsort(g[:, 6])][:, :8]
    b = c[np.argsort(c[:, 6])][:, :8]
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    assert same.all(), f"{(~same).any(axis=1).sum()} rows differ; columns {(~same).sum(axis=0)}"
    return gn


@pytest.mark.parametrize("name", ["drif", "edrift", "kquad_fringe_lossy", "kquad_misaligned", "ksext_k1j1", "koct",
                                  "csbend_k1k2", "csbend_hwang_lindberg", "csbend_rad", "rfca_long", "rfca_tref"])
def test_element_through_hooks_by_do_tracking(name):
    _same_do_tracking(ELEMENT_CASES[name], configs.gaussian_beam(2000, seed=71, sigma_x=1.5e-3, sigma_xp=1.5e-4), 2)


def test_rf_wake_ring_through_hooks_by_do_tracking():
    _same_do_tracking(configs.c2_lattice(cells=4, n_bins=2000), configs.gaussian_beam(3000, seed=72), 3)
    _same_do_tracking(configs.c2_lattice(cells=2, n_bins=500), configs.gaussian_beam(1000, seed=74), 2,
                      pass_offset=4)


def test_lossy_ring_through_hooks_by_do_tracking():
    """Losses on MAXAMP apertures and at elements, and do_tracking's initial
    non-finite screen, which runs before any element."""
    lat = Lattice()
    lat.add("MAXAMP", "AP", X_MAX=0.004, Y_MAX=0.003)
    lat.extend(configs.c1_lattice(cells=2))
    lat.add("MAXAMP", "AP2", X_MAX=0.005, Y_MAX=0.004, ELLIPTICAL=1)
    lat.extend(configs.c1_lattice(cells=2))
    beam = configs.gaussian_beam(3000, seed=73, sigma_x=2e-3, sigma_xp=2e-4)
    beam[5, 0] = np.nan
    beam[9, 1] = 2.0
    assert _same_do_tracking(lat, beam, 3) < beam.shape[0]
