"""CPU pins of the FP64 oracle against outputs of the reference's own CUDA
implementation (tests/golden/ref_tilted_aligned.npz, made by
tests/golden/make_ref_golden.py from the reference sources built for
sm_100a) on the tilted / offset / anisotropic case: the FDK pipeline, the
Joseph pair, the pseudo-matched backprojector and the Siddon pair.

Where the reference interpolates through the texture unit (FDK
backprojection, FP_Joseph, BP_FDK_PseudoMatched) the oracle runs with its
emulation of the 8-bit texture weights.  The bounds are a few times the
residuals measured when the fixtures were made; the residuals are the
reference's FP32 host geometry, incremental stepping and (Siddon) its FP32
face-crossing accumulation.
"""
import os

import numpy as np
import pytest

from tests import cases as K
from tests.golden.make_ref_golden import inputs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_tilted_aligned.npz")


@pytest.fixture(scope="module")
def golden(oracle):
    ref = np.load(GOLDEN)
    case, views, phantom, proj_phantom, smooth, sino = inputs(oracle)
    return ref, case, views, phantom, proj_phantom, smooth, sino


def _check(got, ref, tol):
    err = K.rel_rmse(got, ref)
    assert err <= tol, err


def test_fdk_matches_reference(oracle, golden):
    ref, case, views, phantom, proj_phantom, smooth, sino = golden
    sc = case.scan
    vol = K.oracle_volume(oracle, case.grid)
    _check(oracle.fdk(views, sc.channels, sc.rows, sc.scan_range, vol, oracle.filter_struct(0), smooth),
           ref["fdk_smooth"], 1e-4)
    _check(oracle.fdk(views, sc.channels, sc.rows, sc.scan_range, vol,
                      K.oracle_filter(oracle, case.filt), proj_phantom, flags=1),
           ref["fdk_phantom"], 3e-4)


def test_joseph_pair_matches_reference(oracle, golden):
    ref, case, views, phantom, proj_phantom, smooth, sino = golden
    sc = case.scan
    vol = K.oracle_volume(oracle, case.grid)
    ones = np.ones(case.grid.shape, dtype=np.float32)
    _check(oracle.joseph_fp(views, sc.channels, sc.rows, vol, ones, flags=1),
           ref["fp_joseph_ones"], 1e-4)
    _check(oracle.joseph_bp(views, sc.channels, sc.rows, vol, sino, reference_weight=True),
           ref["bp_joseph"], 1e-4)


def test_pseudo_matched_bp_matches_reference(oracle, golden):
    ref, case, views, phantom, proj_phantom, smooth, sino = golden
    sc = case.scan
    vol = K.oracle_volume(oracle, case.grid)
    _check(oracle.pseudo_bp(views, sc.channels, sc.rows, vol, smooth, tex=True),
           ref["bp_pseudo"], 2e-5)


def test_siddon_pair_matches_reference(oracle, golden):
    ref, case, views, phantom, proj_phantom, smooth, sino = golden
    sc = case.scan
    vol = K.oracle_volume(oracle, case.grid)
    _check(oracle.siddon_fp(views, sc.channels, sc.rows, vol, phantom), ref["fp_siddon"], 5e-5)
    _check(oracle.siddon_bp(views, sc.channels, sc.rows, vol, sino), ref["bp_siddon"], 3e-4)
