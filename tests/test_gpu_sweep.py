"""Harmonic frequency sweep on the resident pattern (eddy currents, hcurl
order 2, harmonics {2,3}).

The drop-in assembles the problem at two fundamental frequencies through
generate()/A(); every term scale and destination multiplier is then fitted as
a + b*omega and the sweep re-processes the resident groups with scales set for
each new frequency.  At a third frequency the result must equal a fresh
generate()/A() of the stock reference at that frequency (same CSR pattern,
values within the drop-in tolerance) and of the drop-in itself.
"""
import numpy as np
import pytest

import _pipeline as P
from sparselizard_b200 import meshgen, workloads as W

pytestmark = pytest.mark.gpu

SIGMAS = [1e3, 5.0e5, 2.0e6, 6.0e7]


def _mesh(tmp_path, n=4):
    rng = np.random.Generator(np.random.PCG64(1))
    tags = meshgen.MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
    msh = str(tmp_path / "e.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=1, element_tags=tags)
    return msh


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("fa", [37.0, 2.5e5])
def test_sweep_matches_fresh_assembly(ref_lib, gpu_lib, tmp_path, fa):
    msh = _mesh(tmp_path)
    got = P.sweep(msh, 2, 1.0e3, 1.0e5, SIGMAS, [1.0, 500.0, fa])
    ref = P.reference(W.EDDY_TET, msh, [2, fa] + SIGMAS)
    dropin = P.gpu(W.EDDY_TET, msh, [2, fa] + SIGMAS)
    for name, other in (("reference", ref), ("drop-in", dropin)):
        assert got["Avals"].size == other["Avals"].size and got["Dvals"].size == other["Dvals"].size
        ea, ed = _rel(got["Avals"], other["Avals"]), _rel(got["Dvals"], other["Dvals"])
        assert ea <= 1e-12 and ed <= 1e-12, f"{name}: relative Frobenius error A {ea:.2e}, D {ed:.2e}"
    assert np.all(got["device_ms"] > 0)
