"""The C++ Session layer (include/ykb_session.hpp) driven by a C++ client
(tests/session_test.cpp) the way YKCBCT's own tests drive its Session."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests import cases as K

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fdk_cuda_impl_b200")


@pytest.fixture(scope="session")
def session_bin(ykb_lib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("session") / "session_test")
    cuda_inc = "/usr/local/cuda/include"
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
           os.path.join(ROOT, "tests", "session_test.cpp"), "-o", out, "-L", PKG, "-lykb",
           f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True)
    return out


def _run(binary, *args, timeout=600):
    res = subprocess.run([binary, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    line = res.stdout.strip().splitlines()[-1] if res.stdout.strip() else "{}"
    return res.returncode, json.loads(line), res.stderr


def test_session_validation_codes(session_bin):
    # status codes of EApiErrorCode before any device work
    rc, out, err = _run(session_bin, "validate")
    assert rc == 0, (out, err)
    assert out["failures"] == 0


@pytest.mark.gpu
def test_session_roundtrip(session_bin, cuda_device):
    # unit_test/test_small_reconstruction.cpp:118-157: cosine > 0.70
    rc, out, err = _run(session_bin, "roundtrip")
    assert rc == 0, (out, err)
    assert out["cosine"] > 0.70


@pytest.mark.gpu
def test_session_streaming(session_bin, cuda_device):
    # dlltest/test_shepp_logan.cpp:158: streamed vs full max diff < 1e-5,
    # cosine > 0.85, NRMSE < 0.65; streaming misuse -> StreamingStateError
    rc, out, err = _run(session_bin, "streaming")
    assert rc == 0, (out, err)
    assert out["failures"] == 0 and out["max_diff"] < 1e-5


@pytest.mark.gpu
def test_session_fdk_and_fp_match_oracle(session_bin, cuda_device, oracle, tmp_path):
    case = K.c1_small()
    sc = case.scan
    views = sc.views()
    ph = K.phantom(oracle, case)
    geo = [sc.total_views, sc.views_per_turn, sc.sid_mm, sc.sdd_mm, sc.channels, sc.rows,
           sc.channel_size_mm, sc.row_size_mm]
    grid = [64, 64, 48, 1.0]
    # forward projection through the Session vs the oracle
    vin, pout = tmp_path / "vol.f32", tmp_path / "proj.f32"
    ph.tofile(vin)
    rc, _, err = _run(session_bin, "fp", vin, pout, *geo, *grid, 1)
    assert rc == 0, err
    proj = np.fromfile(pout, dtype=np.float32).reshape(len(views), sc.rows, sc.channels)
    ref_p = oracle.joseph_fp(views, sc.channels, sc.rows, K.oracle_volume(oracle, case.grid), ph)
    assert K.rel_rmse(proj, ref_p) <= 1e-5
    # EForwardProjector::Automatic resolves to Siddon for a flat detector
    rc, _, err = _run(session_bin, "fp_auto", vin, pout, *geo, *grid, 1)
    assert rc == 0, err
    proj_s = np.fromfile(pout, dtype=np.float32).reshape(len(views), sc.rows, sc.channels)
    ref_s = oracle.siddon_fp(views, sc.channels, sc.rows, K.oracle_volume(oracle, case.grid), ph)
    assert K.rel_rmse(proj_s, ref_s) <= 1e-5
    # FDK through the Session vs the oracle
    pin, vout = tmp_path / "p.f32", tmp_path / "v.f32"
    p32 = ref_p.astype(np.float32)
    p32.tofile(pin)
    rc, _, err = _run(session_bin, "fdk", pin, vout, *geo, *grid, 1)
    assert rc == 0, err
    rec = np.fromfile(vout, dtype=np.float32).reshape(case.grid.shape)
    ref = oracle.fdk(views, sc.channels, sc.rows, sc.scan_range, K.oracle_volume(oracle, case.grid),
                     oracle.filter_struct(1), p32)
    assert K.rel_rmse(rec, ref) <= 1e-5
