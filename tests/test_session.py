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


def _layout(tmp_path, name, includes, defines=()):
    out = str(tmp_path / name)
    cmd = ["g++", "-std=c++17", *defines, *sum((["-I", d] for d in includes), []),
           os.path.join(ROOT, "tests", "session_layout.cpp"), "-o", out]
    subprocess.run(cmd, check=True)
    return subprocess.run([out], capture_output=True, text=True, check=True).stdout


def test_session_header_layout_matches_the_reference(tmp_path):
    # one client source compiles against the reference's public header and
    # against include/ykb_session.hpp; every struct's size, member offsets and
    # scalar defaults, and the enum values, print identically
    from oracle import ref_build
    ours = _layout(tmp_path, "ours", [os.path.join(ROOT, "include"), "/usr/local/cuda/include"])
    assert "sizeof SSystemSpec" in ours and "offsetof SSystemSpec.flat_frame_count" in ours
    if not ref_build.reference_present():
        pytest.skip("reference tree not present (set YKB_REFERENCE_DIR)")
    ref = _layout(tmp_path, "ref", [os.path.join(ref_build.DEFAULT_REFERENCE, "include"),
                                    "/usr/local/cuda/include"], ["-DYKB_LAYOUT_REFERENCE"])
    assert ours == ref


@pytest.mark.gpu
def test_session_caller_frames(session_bin, cuda_device):
    # frames equal to the orbit give the orbit's projections (< 1e-5, the
    # reference's framework/external-geometry pin); the iterative pipelines'
    # request tails are refused by forward projection
    rc, out, err = _run(session_bin, "frames")
    assert rc == 0, (out, err)
    assert out["failures"] == 0 and out["max_diff"] < 1e-5


def _perturbed_frames(views, seed, shift_mm, tilt_rad):
    """The orbit with each view's detector moved in its plane and turned about
    its normal, and the source moved: calibrated geometry of a real scanner."""
    rng = np.random.default_rng(seed)
    f = views.copy()
    for i in range(len(f)):
        u, v = f["detU"][i, :3].astype(np.float64), f["detV"][i, :3].astype(np.float64)
        a = rng.uniform(-tilt_rad, tilt_rad)
        c, s = np.cos(a), np.sin(a)
        f["detU"][i, :3] = c * u + s * v * (np.linalg.norm(u) / np.linalg.norm(v))
        f["detV"][i, :3] = -s * u * (np.linalg.norm(v) / np.linalg.norm(u)) + c * v
        f["detS"][i, :3] += rng.uniform(-shift_mm, shift_mm) * (u / np.linalg.norm(u)) + \
            rng.uniform(-shift_mm, shift_mm) * (v / np.linalg.norm(v))
        f["src"][i, :3] += rng.uniform(-shift_mm, shift_mm, 3)
    return np.ascontiguousarray(f)


@pytest.mark.gpu
def test_session_caller_frames_match_oracle(session_bin, cuda_device, oracle, tmp_path):
    # forward projection accepts any frames; FDK accepts frames within 1e-3
    # of the orbit (src/interface/YkReconstructionApi.cpp:146-168) and then
    # reconstructs with them; both against the FP64 oracle on the same frames
    case = K.c1_small()
    sc = case.scan
    views = sc.views()
    ph = K.phantom(oracle, case)
    geo = [sc.total_views, sc.views_per_turn, sc.sid_mm, sc.sdd_mm, sc.channels, sc.rows,
           sc.channel_size_mm, sc.row_size_mm]
    grid = [64, 64, 48, 1.0]
    ovol = K.oracle_volume(oracle, case.grid)
    vin, pout, fpath = tmp_path / "vol.f32", tmp_path / "proj.f32", tmp_path / "frames.bin"
    ph.tofile(vin)
    calibrated = _perturbed_frames(views, 5, 1.5, 0.02)
    calibrated.tofile(fpath)
    rc, _, err = _run(session_bin, "fp", vin, pout, *geo, *grid, 1, fpath)
    assert rc == 0, err
    proj = np.fromfile(pout, dtype=np.float32).reshape(len(views), sc.rows, sc.channels)
    ref_p = oracle.joseph_fp(calibrated, sc.channels, sc.rows, ovol, ph)
    assert K.rel_rmse(proj, ref_p) <= 1e-5
    # the orbit's own projections differ: the frames were used
    orbit_p = oracle.joseph_fp(views, sc.channels, sc.rows, ovol, ph)
    assert K.rel_rmse(orbit_p, ref_p) > 1e-3
    # FDK with frames 0.5 um off the orbit
    near = _perturbed_frames(views, 6, 5e-4, 0.0)
    near.tofile(fpath)
    pin, vout = tmp_path / "p.f32", tmp_path / "v.f32"
    p32 = orbit_p.astype(np.float32)
    p32.tofile(pin)
    rc, _, err = _run(session_bin, "fdk", pin, vout, *geo, *grid, 1, fpath)
    assert rc == 0, err
    rec = np.fromfile(vout, dtype=np.float32).reshape(case.grid.shape)
    ref = oracle.fdk(near, sc.channels, sc.rows, sc.scan_range, ovol, oracle.filter_struct(1), p32)
    assert K.rel_rmse(rec, ref) <= 1e-5
