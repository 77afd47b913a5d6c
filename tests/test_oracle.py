"""CPU tests of the FP64 oracle: geometry conventions, closed forms, the
reference test-suite's pins, and the restatement's internal consistency."""
import numpy as np
import pytest

from tests import cases as K


def test_zero_angle_geometry_convention(oracle):
    # doc/geometry-and-data.md:9-17: source (0,-SID,z), principal point
    # (0,SDD-SID,z), U=(+1,0,0), V=(0,0,+1); detS = pixel (0,0) centre
    v = oracle.build_circular_flat(4, 4, 500.0, 1000.0, 192, 128, 0.8, 0.8, z=3.0)[0]
    assert np.allclose(v["src"][:3], [0, -500, 3], atol=1e-5)
    assert np.allclose(v["detU"][:3], [0.8, 0, 0], atol=1e-7)
    assert np.allclose(v["detV"][:3], [0, 0, 0.8], atol=1e-7)
    centre = v["detS"][:3] + 95.5 * v["detU"][:3] + 63.5 * v["detV"][:3]
    assert np.allclose(centre, [0, 500, 3], atol=1e-4)


def test_rotation_direction_and_range(oracle):
    a = oracle.build_circular_flat(8, 8, 100.0, 200.0, 8, 8, 1.0, 1.0)
    b = oracle.build_circular_flat(8, 8, 100.0, 200.0, 8, 8, 1.0, 1.0, direction=-1)
    assert np.isclose(a["angle"][1, 0], 2 * np.pi / 8, rtol=1e-6)
    assert np.isclose(b["angle"][1, 0], -2 * np.pi / 8, rtol=1e-6)
    # views_per_turn < total_views: multi-turn range
    assert np.isclose(oracle.regular_scan_range(720, 360), 4 * np.pi, rtol=1e-6)


def test_derived_centred_geometry(oracle):
    v = oracle.build_circular_flat(12, 12, 500.0, 1000.0, 192, 128, 0.8, 0.8)
    d = oracle.fdk_derived(v, 192, 128, oracle.regular_scan_range(12, 12))
    assert np.allclose(d[:, 3], 500.0, rtol=1e-6)   # SID
    assert np.allclose(d[:, 4], 1000.0, rtol=1e-6)  # DSD
    assert np.allclose(d[:, 5], 1000.0, rtol=1e-6)  # plane distance
    assert np.allclose(d[:, 6:8], 0.0, atol=1e-3)   # principal point offsets
    assert np.allclose(d[:, 1], 2 * np.pi / 12, rtol=1e-6)  # dtheta
    assert np.allclose(d[:, 2], 1.0, rtol=1e-6)     # 2pi / range
    # startU = lrint(N/2 - (Nu-1)/2): N = 512 for Nu = 192
    assert np.all(d[:, 10] == np.rint(256 - 95.5))


def test_ramlak_closed_form(oracle):
    # band-limited ramp (Kak & Slaney, Principles of CT Imaging, eq. 3.61):
    # h(0) = 1/(4 du^2) du, h(odd n) = -1/(pi^2 n^2 du), h(even n) = 0,
    # approached by the length-N analytic frequency weights.
    nu, du = 256, 0.8
    h = oracle.ramp_kernel(nu, du, oracle.filter_struct(1))
    c = nu - 1
    assert np.isclose(h[c], 1.0 / (4 * du), rtol=1e-12)
    n = np.arange(1, 40)
    ref = np.where(n % 2 == 1, -1.0 / (np.pi ** 2 * n ** 2 * du), 0.0)
    assert np.allclose(h[c + n], ref, atol=2e-4 / du)
    assert np.allclose(h[c + n], h[c - n])


def _numpy_window(x, kind):
    x = np.clip(x, 0, 1)
    return {1: np.ones_like(x), 2: np.sinc(0.5 * x), 3: np.cos(0.5 * np.pi * x),
            4: 0.5 * (1 + np.cos(np.pi * x)), 5: 0.54 + 0.46 * np.cos(np.pi * x),
            6: 0.42 + 0.5 * np.cos(np.pi * x) + 0.08 * np.cos(2 * np.pi * x),
            7: 1.0 / (1.0 + x ** 4)}[kind]


@pytest.mark.parametrize("kind", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("cutoff", [0.5, 0.35])
def test_ramp_kernel_matches_irfft_and_dc_is_zero(oracle, kind, cutoff):
    # The padded FFT filter of the reference (pad to N = 2^ceil(log2 2nu),
    # R2C, multiply by w[k] = f*window(f/cutoff)/N/du for f = k/N <= cutoff,
    # C2R) equals a Toeplitz convolution with h = N * irfft(w) on |lag| < nu.
    # The DC weight is zero, so the full-period kernel sums to zero
    # (filter/discrete-ramlak-dc, Yktest/test_filter_validation.cpp:17-46).
    nu, du = 100, 0.7
    N = 256
    cutoff = float(np.float32(cutoff))  # the C struct holds float
    f = np.arange(N // 2 + 1) / N
    w = np.where(f <= cutoff, f * _numpy_window(f / cutoff, kind) / du, 0.0)
    full = np.fft.irfft(w, n=N)
    assert abs(full.sum()) < 1e-12 * np.abs(full).max() * N
    h = oracle.ramp_kernel(nu, du, oracle.filter_struct(kind, cutoff=cutoff, order=2.0))
    lags = np.arange(-(nu - 1), nu)
    assert np.allclose(h, full[lags % N], rtol=1e-9, atol=1e-12)


def test_oracle_adjoint_fp64(oracle):
    case = K.c1_small()
    views = case.scan.views()
    vol = K.oracle_volume(oracle, case.grid)
    x = oracle.uniform(case.grid.shape, 0.0, 1.0, 11)
    y = oracle.normal((len(views), case.scan.rows, case.scan.channels), 12)
    ax = oracle.joseph_fp(views, case.scan.channels, case.scan.rows, vol, x)
    aty = oracle.joseph_bp(views, case.scan.channels, case.scan.rows, vol, y)
    lhs, rhs = float((ax * y).sum()), float((x * aty).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_oracle_bp_reference_weight_isotropic(oracle):
    # for isotropic voxels the reference's BP_Joseph factor vox0*sqrt(1+a1^2+a2^2)
    # equals the forward chord length, so both backprojections coincide
    case = K.c1_small()
    views = case.scan.views()
    vol = K.oracle_volume(oracle, case.grid)
    y = oracle.normal((len(views), case.scan.rows, case.scan.channels), 5)
    a = oracle.joseph_bp(views, case.scan.channels, case.scan.rows, vol, y)
    b = oracle.joseph_bp(views, case.scan.channels, case.scan.rows, vol, y, reference_weight=True)
    assert K.rel_rmse(b, a) < 1e-12


def test_small_reconstruction_pin(oracle):
    # unit_test/test_small_reconstruction.cpp:118-157: FP(Joseph) -> FDK on a
    # 24x24x16 grid, 96 views, 48x32 detector, SID/SDD 100/200 mm; cosine > 0.70
    scan_views = oracle.build_circular_flat(96, 96, 100.0, 200.0, 48, 32, 1.0, 1.0)
    vol = oracle.volume_struct((16, 24, 24), 1.0)
    E = oracle.Ellipsoid
    truth = oracle.voxelize(vol, [E(0, 0, 0, 7, 8, 5, 0, 0, 0, 0.02),
                                  E(3, -2, 0, 1.5, 1.5, 1.5, 0, 0, 0, 0.04)])
    p = oracle.joseph_fp(scan_views, 48, 32, vol, truth).astype(np.float32)
    rec = oracle.fdk(scan_views, 48, 32, oracle.regular_scan_range(96, 96), vol,
                     oracle.filter_struct(1), p)
    assert rec.max() > 0
    assert K.cosine(rec, truth) > 0.70


def test_dll_smoke_pin(oracle):
    # dlltest/test_shepp_logan.cpp:32-51,158 thresholds (cosine > 0.85,
    # NRMSE < 0.65) on its geometry: 64^3 @ 0.75 mm, 128^2 @ 0.8 mm, 360
    # views, SID/SDD 200/400, Ram-Lak; a seeded ellipsoid phantom stands in
    # for the test's phantom.
    views = oracle.build_circular_flat(360, 360, 200.0, 400.0, 128, 128, 0.8, 0.8)
    vol = oracle.volume_struct((64, 64, 64), 0.75)
    truth = oracle.voxelize(vol, oracle.random_ellipsoids(3, 10, 8.0, 2.0, 14.0, 0.0, 0.02))
    p = oracle.joseph_fp(views, 128, 128, vol, truth).astype(np.float32)
    rec = oracle.fdk(views, 128, 128, oracle.regular_scan_range(360, 360), vol,
                     oracle.filter_struct(1), p)
    nrmse = np.sqrt(np.mean((rec - truth) ** 2)) / np.sqrt(np.mean(truth.astype(np.float64) ** 2))
    assert K.cosine(rec, truth) > 0.85
    assert nrmse < 0.65


def test_oracle_fdk_batch_linearity(oracle):
    # streaming FDK: the sum of the views' contributions equals the full run
    case = K.c1_small()
    views = case.scan.views()
    p = K.projections(oracle, case, views)
    vol = K.oracle_volume(oracle, case.grid)
    rng = case.scan.scan_range
    f = oracle.fdk_filter(views, 96, 64, rng, K.oracle_filter(oracle, case.filt), p)
    full = oracle.fdk_backproject(views, 96, 64, rng, vol, f)
    a = oracle.fdk_backproject(views, 96, 64, rng, vol, f)  # same call twice is deterministic
    assert np.array_equal(full, a)


def test_texture_emulation_bounded(oracle):
    case = K.c1_small()
    views = case.scan.views()
    p = K.projections(oracle, case, views)
    vol = K.oracle_volume(oracle, case.grid)
    f = K.oracle_filter(oracle, case.filt)
    exact = oracle.fdk(views, 96, 64, case.scan.scan_range, vol, f, p)
    tex = oracle.fdk(views, 96, 64, case.scan.scan_range, vol, f, p, flags=1)
    err = K.rel_rmse(tex, exact)
    assert 1e-7 < err < 5e-3


def test_fp32_transcription_within_budget(oracle):
    case = K.c1_small()
    views = case.scan.views()
    p = K.projections(oracle, case, views)
    vol = K.oracle_volume(oracle, case.grid)
    f = K.oracle_filter(oracle, case.filt)
    exact = oracle.fdk(views, 96, 64, case.scan.scan_range, vol, f, p)
    f32 = oracle.fdk_fp32(views, 96, 64, case.scan.scan_range, vol, f, p)
    assert K.rel_rmse(f32, exact) < 1e-5


def test_poisson_noise_statistics(oracle):
    p = np.full(200000, 2.0, dtype=np.float32)
    i0 = 1e5
    noisy = oracle.poisson_noise(p, i0, 9)
    counts = i0 * np.exp(-noisy.astype(np.float64))
    lam = i0 * np.exp(-2.0)
    assert abs(counts.mean() / lam - 1) < 2e-3
    assert abs(counts.var() / lam - 1) < 3e-2
    # deterministic per seed, independent of thread count
    oracle.set_num_threads(1)
    again = oracle.poisson_noise(p, i0, 9)
    oracle.set_num_threads(oracle.num_threads())
    assert np.array_equal(noisy, again)


def test_mt19937_stream_matches_reference_generator(oracle):
    # std::mt19937(12345) + uniform_real_distribution<float>(-1,1) as the
    # reference adjoint test draws it (unit_test/test_operator_benchmarks.cpp:466-473)
    x = oracle.mt19937_uniform_pm1(1000, 12345)
    assert x.min() >= -1 and x.max() < 1
    assert abs(x.mean()) < 0.1
    assert not np.array_equal(x, oracle.mt19937_uniform_pm1(1000, 54321))


# ---------------------------------------------------------------- Parker ---

def _short_case(total=40, per_turn=60):
    from fdk_cuda_impl_b200.geometry import CircularScan
    case = K.c1_small()
    case.scan = CircularScan(total, per_turn, 500.0, 1000.0, 96, 64, 1.6, 1.6)
    return case


def test_parker_conjugate_rays_sum_to_one(oracle):
    # w(beta, gamma) + w(beta + pi + 2 gamma, -gamma) = 1 (before the range/pi
    # scale): on the central column (gamma = 0, odd detector, no offsets) of a
    # scan sampled every 0.9 degrees the conjugate of view i is view i + 200
    # (YkFDKParkerKernels.cu:46-110; the Parker 1982 condition)
    from fdk_cuda_impl_b200.geometry import CircularScan
    sc = CircularScan(260, 400, 500.0, 1000.0, 97, 8, 1.6, 1.6)
    views = sc.views()
    w = oracle.parker_weights(views, 97, 8, sc.scan_range)
    scale = sc.scan_range / np.pi
    c = w[:, 48] / scale
    assert np.all((w >= 0) & (w <= scale + 1e-12))
    pairs = c[:60] + c[200:260]
    # the view angles are floats (ulp 5e-7 rad at 4 rad)
    assert np.max(np.abs(pairs - 1.0)) < 1e-5
    assert c[0] == 0.0 and np.all(c[80:120] == 1.0)


def test_parker_needs_a_qualifying_short_scan(oracle):
    from fdk_cuda_impl_b200.geometry import CircularScan
    full = CircularScan(60, 60, 500.0, 1000.0, 96, 64, 1.6, 1.6)
    with pytest.raises(RuntimeError):
        oracle.parker_weights(full.views(), 96, 64, full.scan_range)
    # 180 degrees do not cover pi + 2 x fan angle (fan half-angle 4.4 degrees)
    short = CircularScan(30, 60, 500.0, 1000.0, 96, 64, 1.6, 1.6)
    with pytest.raises(RuntimeError):
        oracle.parker_weights(short.views(), 96, 64, short.scan_range)


def test_short_scan_fdk_matches_full_scan(oracle):
    # Parker-weighted short scan (240 of 360 degrees) reconstructs the same
    # object as the full scan: the weights and the range/pi x 2pi/range
    # normalisation pin the short-scan path
    full = K.c1_small()
    short = _short_case()
    ph = K.phantom(oracle, full)
    vol = K.oracle_volume(oracle, full.grid)
    filt = K.oracle_filter(oracle, full.filt)
    pf = K.projections(oracle, full, ph=ph)
    ref = oracle.fdk(full.scan.views(), 96, 64, full.scan.scan_range, vol, filt, pf)
    sv = short.scan.views()
    ps = K.projections(oracle, short, ph=ph)
    w = oracle.parker_weights(sv, 96, 64, short.scan.scan_range)
    rec = oracle.fdk_weighted(sv, 96, 64, short.scan.scan_range, vol, filt, ps, w)
    assert K.cosine(rec, ref) > 0.99
    assert K.rel_rmse(rec, ref) < 0.15
    # without the weights the short scan is visibly wrong
    plain = oracle.fdk(sv, 96, 64, short.scan.scan_range, vol, filt, ps)
    assert K.rel_rmse(plain, ref) > 2 * K.rel_rmse(rec, ref)


@pytest.mark.parametrize("smooth", [False, True])
def test_pseudo_bp_transposes_the_projector_on_smooth_data(oracle, smooth):
    # BP_FDK_PseudoMatched weights each voxel by the ray density of the
    # line-integral projector (voxel volume x L^3 / (|P-S|^2 SDD_plane du dv)),
    # so it is the transpose of the Joseph projector up to the interpolation
    # kernel: on slowly varying data <A x, y> = <x, B y> to a few 1e-4.
    from tests import cases as K
    case = K.c1_small()
    views = case.scan.views()
    nu, nv = case.scan.channels, case.scan.rows
    vol = K.oracle_volume(oracle, case.grid)
    x = oracle.uniform(case.grid.shape, 0.0, 1.0, 5)
    if smooth:
        u = np.arange(nu)[None, None, :] / nu
        v = np.arange(nv)[None, :, None] / nv
        k = np.arange(len(views))[:, None, None] / len(views)
        y = (1.0 + 0.3 * np.cos(np.pi * u) * np.sin(np.pi * v) + 0.2 * np.cos(2 * np.pi * k))
        y = np.ascontiguousarray(np.broadcast_to(y, (len(views), nv, nu)), dtype=np.float32)
    else:
        y = np.ones((len(views), nv, nu), dtype=np.float32)
    lhs = float((oracle.joseph_fp(views, nu, nv, vol, x) * y).sum())
    rhs = float((x * oracle.pseudo_bp(views, nu, nv, vol, y)).sum())
    assert abs(lhs - rhs) / abs(lhs) < 2e-3


@pytest.mark.parametrize("case_fn", [K.c1_small, K.odd_case])
def test_siddon_oracle_pins(oracle, case_fn):
    # FP of a constant volume is the chord of the ray through the volume box
    # (slab clipping in numpy, independent of the oracle's voxel walk); the
    # backprojector is the exact transpose (the reference's Siddon adjoint
    # error bound is 1e-4, unit_test/test_operator_benchmarks.cpp:978)
    case = case_fn()
    views = case.scan.views()
    nu, nv = case.scan.channels, case.scan.rows
    g = case.grid
    vol = K.oracle_volume(oracle, g)
    ones = np.ones(g.shape, dtype=np.float32)
    got = oracle.siddon_fp(views, nu, nv, vol, ones)
    n = np.array([g.nx, g.ny, g.nz], dtype=np.float64)
    # the grid as the volume struct holds it (float members)
    vox = np.array(g.voxel_mm, dtype=np.float32).astype(np.float64)
    lo = np.array(g.center_mm, dtype=np.float32).astype(np.float64) - 0.5 * n * vox
    hi = lo + n * vox
    iu, iv = np.meshgrid(np.arange(nu), np.arange(nv))
    chord = np.zeros((len(views), nv, nu))
    for k, vw in enumerate(views):
        s = vw["src"][:3].astype(np.float64)
        d = (vw["detS"][:3].astype(np.float64) + iu[..., None] * vw["detU"][:3].astype(np.float64)
             + iv[..., None] * vw["detV"][:3].astype(np.float64))
        r = d - s
        with np.errstate(divide="ignore", invalid="ignore"):
            ta, tb = (lo - s) / r, (hi - s) / r
        tmin = np.clip(np.max(np.minimum(ta, tb), axis=-1), 0.0, None)
        tmax = np.clip(np.min(np.maximum(ta, tb), axis=-1), None, 1.0)
        chord[k] = np.clip(tmax - tmin, 0.0, None) * np.linalg.norm(r, axis=-1)
    assert np.abs(got - chord).max() <= 1e-9 * chord.max()
    x = oracle.uniform(g.shape, 0.0, 1.0, 5)
    y = oracle.normal((len(views), nv, nu), 6)
    lhs = float((oracle.siddon_fp(views, nu, nv, vol, x) * y).sum())
    rhs = float((x * oracle.siddon_bp(views, nu, nv, vol, y)).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("case_fn,slabs", [(K.c1_small, [(0.0, 4), (14.0, 6), (-20.5, 3)]),
                                           (K.odd_case, [(0.75, 3), (4.0, 2)])])
def test_row_band_fdk_equals_full_detector(oracle, case_fn, slabs):
    # the oracle slabs of the full-size workloads filter and backproject only
    # the detector rows a few slices read; the result must equal the full
    # detector's bit for bit (the filter acts on rows alone, and the band
    # holds every row of each voxel's bilinear footprint)
    case = case_fn()
    views = case.scan.views()
    nu, nv = case.scan.channels, case.scan.rows
    p = K.projections(oracle, case, views)
    f = K.oracle_filter(oracle, case.filt)
    g = case.grid
    for zc, nz in slabs:
        vol = oracle.volume_struct((nz, g.ny, g.nx), g.voxel_mm,
                                   (g.center_mm[0], g.center_mm[1], zc))
        r0, nr = oracle.fdk_row_band(views, nu, nv, case.scan.scan_range, vol)
        assert 0 < nr < nv
        full = oracle.fdk(views, nu, nv, case.scan.scan_range, vol, f, p)
        band = oracle.fdk_rows(views, nu, nv, case.scan.scan_range, vol, f, p[:, r0:r0 + nr], r0)
        assert np.array_equal(full, band)
