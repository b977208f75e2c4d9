"""Pins the C restatement oracle to the reference itself (no GPU needed).

The drop-in lowers each workload on a record-only context (no device); the
oracle assembles the recorded groups on the CPU; the result must match
stock sparselizard's generate()/A()/b() on the same mesh: CSR pattern
bit-exact, values within 1e-12 row-relative (the reference's DGEMM sums in a
different order, so bit equality of values is not expected), b on the
unconstrained DOFs (the reference's b() writes Dirichlet values afterwards).
"""
import os

import numpy as np
import pytest

import _pipeline as P
from sparselizard_b200 import meshgen, workloads as W

TOL = 1e-12


@pytest.fixture(scope="module")
def tmp(tmp_path_factory):
    return tmp_path_factory.mktemp("meshes")


def _pin(ref, rec):
    P.check_pattern(ref, rec)
    errs = P.check_values(ref, rec, TOL, mag=rec)
    if "b_raw" in rec:
        P.check_rhs(ref, rec["b_raw"], TOL, unconstrained_only=True, babs=rec["b_abs"])
    return errs


def test_poisson_quad_order1(ref_lib, gpu_lib, tmp):
    msh = str(tmp / "q.msh")
    meshgen.quad_mesh(msh, 24, jitter=0.2, seed=1)
    ref = P.reference(W.POISSON_QUAD, msh, [1])
    rec = P.record_oracle(W.POISSON_QUAD, msh, [1])
    _pin(ref, rec)
    assert ref["Acols"].size > 0 and ref["Dcols"].size > 0


@pytest.mark.parametrize("order", [2, 3])
def test_poisson_quad_high_order(ref_lib, gpu_lib, tmp, order):
    msh = str(tmp / f"q{order}.msh")
    meshgen.quad_mesh(msh, 10, jitter=0.2, seed=3)
    ref = P.reference(W.POISSON_QUAD, msh, [order])
    rec = P.record_oracle(W.POISSON_QUAD, msh, [order])
    _pin(ref, rec)


def test_elasticity_hex_order2(ref_lib, gpu_lib, tmp):
    msh = str(tmp / "h.msh")
    meshgen.hex_mesh(msh, 3, jitter=0.15, seed=1)
    ref = P.reference(W.ELASTICITY_HEX, msh, [2, -2])
    rec = P.record_oracle(W.ELASTICITY_HEX, msh, [2, -2])
    _pin(ref, rec)


def test_helmholtz_tet_p_adaptive(ref_lib, gpu_lib, tmp):
    n = 3
    rng = np.random.Generator(np.random.PCG64(7))
    tags = meshgen.ORDER_REGION_BASE + rng.integers(1, 6, size=6 * n ** 3)
    msh = str(tmp / "t.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=2, element_tags=tags)
    ref = P.reference(W.HELMHOLTZ_TET, msh, [])
    rec = P.record_oracle(W.HELMHOLTZ_TET, msh, [])
    _pin(ref, rec)


def test_eddy_hcurl_harmonic(ref_lib, gpu_lib, tmp):
    n = 2
    rng = np.random.Generator(np.random.PCG64(11))
    tags = meshgen.MATERIAL_REGION_BASE + rng.integers(0, 4, size=6 * n ** 3)
    msh = str(tmp / "e.msh")
    meshgen.tet_mesh(msh, n, jitter=0.1, seed=4, element_tags=tags)
    sig = [1e3, 5e5, 2e6, 6e7]
    ref = P.reference(W.EDDY_TET, msh, [2, 1000.0] + sig)
    rec = P.record_oracle(W.EDDY_TET, msh, [2, 1000.0] + sig)
    _pin(ref, rec)
