"""Pins the CPU FP64 oracle against the reference's own tests for this path.

The reference (a Julia package) cannot run in this container, so the oracle is checked against
what its test-suite fixes: brute-force all-pairs sums, closed-form properties, and the numeric
known-answer values it asserts.  Each test names the reference test it restates; grids follow
the reference's (1-based Julia indices are converted to 0-based here).  No GPU is needed.
"""
import math

import numpy as np
import pytest

import oracle as O
from fields import fourier_slope, logfit, spectral_field

R_EARTH = 6.371e6


def haversine(R, lon1, lat1, lon2, lat2):
    h = np.sin((lat2 - lat1) / 2) ** 2 + np.cos(lat1) * np.cos(lat2) * np.sin((lon2 - lon1) / 2) ** 2
    return 2 * R * np.arcsin(np.sqrt(np.minimum(h, 1.0)))


# ---------------------------------------------------------------------------------------------
# test/test_filtering.jl:733-768 -- banded spherical footprint vs an all-pairs brute force at high
# latitude, where the ball reaches over the pole (window must cover it, ring counted once).
# ---------------------------------------------------------------------------------------------
def test_sphere_footprint_matches_all_pairs_brute_force_over_the_pole():
    nlat, nlon = 60, 120
    lat0, dlat = -math.pi / 2 + 1e-6, (math.pi - 2e-6) / (nlat - 1)
    g = O.Grid(O.SPHERE, nlon, nlat, 0.0, 2 * math.pi / nlon, lat0, dlat, R_EARTH, True, False)
    alpha, scale = 6.0, 3.0e6
    rad = O.kernel_radius(O.GAUSSIAN, alpha, scale)
    assert rad > R_EARTH * (math.pi / 2 - 1.33)
    p = O.Plan(g, O.GAUSSIAN, alpha, scale)
    assert p.engine == O.ENGINE_BANDED
    lon, lat = p.coords()
    LON, LAT = np.meshgrid(lon, lat)  # (ny, nx)
    fld = np.cos(3 * LON) * np.exp(-(((np.abs(LAT) - 1.40) / 0.12) ** 2))
    out = p.filter(fld)
    area = R_EARTH ** 2 * np.cos(LAT) * g.dx * g.dy
    for j in (2, 4, nlat - 6, nlat - 3, nlat - 1):
        for i in (1, 37):
            jj, ii = j - 1, i - 1
            d = haversine(R_EARTH, lon[ii], lat[jj], LON, LAT)
            sel = d <= rad
            wgt = np.exp(-alpha * (d[sel] / scale) ** 2) * area[sel]
            ref = np.sum(wgt * fld[sel]) / np.sum(wgt)
            assert out[jj, ii] == pytest.approx(ref, rel=1e-12)


# ---------------------------------------------------------------------------------------------
# test/test_periodic.jl:3-82 -- periodic sphere top-hat (prefix-sum engine) vs an area-weighted
# all-pairs average; the seam wraps, and a non-periodic copy loses the wrapped band.
# ---------------------------------------------------------------------------------------------
def test_periodic_sphere_tophat_matches_brute_force_and_wraps_the_seam():
    lon_deg = np.arange(0.0, 356.0, 5.0)
    lat_deg = np.arange(-45.0, 46.0, 5.0)
    nx, ny = len(lon_deg), len(lat_deg)
    d5 = math.radians(5.0)
    g = O.Grid(O.SPHERE, nx, ny, 0.0, d5, math.radians(-45.0), d5, R_EARTH, True, False)
    field = np.zeros((ny, nx))
    field[:, (lon_deg > 350.0) | (lon_deg < 10.0)] = 1.0
    # The reference's radius (10 degrees of arc) falls exactly on grid columns, where inclusion is
    # decided by the last ulp of two different formulas (haversine vs the acos band); widen it by
    # 1e-9 so every boundary column is unambiguously inside, as the reference's test intends.
    scale = math.radians(20.0) * R_EARTH * (1 + 1e-9)
    p = O.Plan(g, O.TOPHAT, 0.0, scale)
    assert p.engine == O.ENGINE_PREFIXSUM
    out = p.filter(field)
    lon, lat = p.coords()
    LON, LAT = np.meshgrid(lon, lat)
    rad = O.kernel_radius(O.TOPHAT, 0.0, scale)
    area = R_EARTH ** 2 * np.cos(LAT) * d5 * d5

    def brute(i0, j0):
        d = haversine(R_EARTH, lon[i0], lat[j0], LON, LAT)
        sel = d <= rad
        return np.sum(field[sel] * area[sel]) / np.sum(area[sel])

    j10 = 9
    assert out[j10, 0] == pytest.approx(brute(0, j10), rel=1e-10)
    assert out[j10, nx - 1] == pytest.approx(brute(nx - 1, j10), rel=1e-10)
    i30 = int(np.where(lon_deg == 30.0)[0][0])
    assert out[j10, i30] == pytest.approx(brute(i30, j10), rel=1e-10)
    assert out[j10, i30] < out[j10, 0]
    gnp = O.Grid(O.SPHERE, nx, ny, 0.0, d5, math.radians(-45.0), d5, R_EARTH, False, False)
    assert out[j10, nx - 1] == pytest.approx(out[j10, 1], rel=1e-12)  # mirror image across the seam
    out_np = O.Plan(gnp, O.TOPHAT, 0.0, scale).filter(field)
    assert out_np[j10, nx - 1] < out[j10, nx - 1]


# ---------------------------------------------------------------------------------------------
# test/test_filtering.jl:472-550 -- separable fast path vs a brute-force square-truncated sum,
# masked, anisotropic spacing, both mask strategies.
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("strategy", [O.ZEROFILL, O.DEFORMABLE])
def test_separable_matches_square_truncated_brute_force(strategy):
    N = 24
    dx, dy, alpha, scale = 1000.0, 1500.0, 6.0, 4000.0
    mask = np.ones((N, N), bool)
    mask[7:11, 7:11] = False   # Julia mask[8:11, 8:11]
    mask[:, 0] = False         # Julia mask[1, :] (first x index, every y)
    g = O.Grid(O.CART, N, N, 0.0, dx, 0.0, dy, mask=mask)
    p = O.Plan(g, O.GAUSSIAN, alpha, scale, strategy)
    assert p.engine == O.ENGINE_SEPARABLE
    I, J = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1))  # Julia i (x), j (y)
    field = np.sin(I / 3.0) * np.cos(J / 4.0)
    out = p.filter(field)
    rad = O.kernel_radius(O.GAUSSIAN, alpha, scale)
    dil, djl = math.ceil(rad / dx), math.ceil(rad / dy)
    gx = np.exp(-alpha * ((np.arange(-dil, dil + 1) * dx) / scale) ** 2)
    gy = np.exp(-alpha * ((np.arange(-djl, djl + 1) * dy) / scale) ** 2)
    ref = np.zeros((N, N))
    for j in range(N):
        for i in range(N):
            if not mask[j, i]:
                continue
            ws = wn = 0.0
            for ddj in range(-djl, djl + 1):
                for ddi in range(-dil, dil + 1):
                    ii, jj = i + ddi, j + ddj
                    if not (0 <= ii < N and 0 <= jj < N):
                        continue
                    w = gx[ddi + dil] * gy[ddj + djl]
                    if strategy == O.ZEROFILL:
                        wn += w
                        if mask[jj, ii]:
                            ws += w * field[jj, ii]
                    elif mask[jj, ii]:
                        wn += w
                        ws += w * field[jj, ii]
            ref[j, i] = ws / wn if wn > 1e-15 else 0.0
    np.testing.assert_allclose(out, ref, rtol=1e-10, atol=0)


# ---------------------------------------------------------------------------------------------
# test/test_filtering.jl:698-731 -- a constant filters to the constant in the interior.
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("kernel", [O.TOPHAT, O.GAUSSIAN])
@pytest.mark.parametrize("scale", [5000.0, 10000.0, 20000.0])
def test_constant_field_is_preserved(kernel, scale):
    n = 51
    g = O.Grid(O.CART, n, n, 0.0, 1000.0, 0.0, 1000.0)
    C = 42.0
    for strategy in (O.ZEROFILL, O.DEFORMABLE):
        out = O.Plan(g, kernel, 6.0, scale, strategy).filter(np.full((n, n), C))
        np.testing.assert_allclose(out[19:n - 20, 19:n - 20], C, rtol=1e-10)


# ---------------------------------------------------------------------------------------------
# test/test_filtering.jl:850-916 -- ZeroFill commutes with d/dx, Deformable does not; ZeroFill
# conserves the domain integral.
# ---------------------------------------------------------------------------------------------
def _bump(N, ic, jc, rad):
    I, J = np.meshgrid(np.arange(1, N + 1), np.arange(1, N + 1))
    r2 = ((I - ic) ** 2 + (J - jc) ** 2) / rad ** 2
    return np.where(r2 < 1, (1 - r2) ** 4, 0.0)


def test_zerofill_commutes_with_ddx_and_deformable_does_not():
    N, dx, icoast, ell = 96, 1000.0, 61, 8000.0
    mask = np.ones((N, N), bool)
    mask[:, icoast - 1:] = False
    g = O.Grid(O.CART, N, N, 0.0, dx, 0.0, dx, mask=mask)
    f = _bump(N, 49, 48, 8)
    pz = O.Plan(g, O.TOPHAT, 0.0, ell, O.ZEROFILL)
    df = pz.ddx(f)
    assert np.all(f[:, icoast - 1:] == 0) and np.all(df[:, icoast - 1:] == 0)
    rel, edge, drift = {}, {}, {}
    for strat in (O.ZEROFILL, O.DEFORMABLE):
        p = O.Plan(g, O.TOPHAT, 0.0, ell, strat)
        lhs = p.filter(df)
        ff = p.filter(f)
        rhs = p.ddx(ff)
        ii = slice(1, icoast - 2)  # Julia 2:(icoast-2)
        s = np.max(np.abs(rhs[:, ii]))
        rel[strat] = np.max(np.abs(lhs[:, ii] - rhs[:, ii])) / s
        edge[strat] = np.max(np.abs(lhs[:, icoast - 2] - rhs[:, icoast - 2])) / s
        drift[strat] = (ff.sum() - f.sum()) / f.sum()
    assert rel[O.ZEROFILL] < 1e-13
    assert rel[O.DEFORMABLE] > 1e-3
    assert rel[O.DEFORMABLE] > 1e9 * rel[O.ZEROFILL]
    assert edge[O.ZEROFILL] > 1e-3
    assert abs(drift[O.ZEROFILL]) < 1e-13
    assert abs(drift[O.DEFORMABLE]) > 1e-6
    # Unmasked: both kernels commute.
    gf = O.Grid(O.CART, N, N, 0.0, dx, 0.0, dx)
    fu = _bump(N, 48, 48, 10)
    for kern in (O.TOPHAT, O.GAUSSIAN):
        p = O.Plan(gf, kern, 6.0, ell)
        lhs = p.filter(p.ddx(fu))
        rhs = p.ddx(p.filter(fu))
        ii = slice(1, N - 1)
        assert np.max(np.abs(lhs[:, ii] - rhs[:, ii])) < 1e-13 * np.max(np.abs(rhs[:, ii]))


# ---------------------------------------------------------------------------------------------
# test/test_filtering.jl:918-961 -- the coast known-answer values (Gaussian alpha=6, l=16 cells,
# coast at column 101 of 200).
# ---------------------------------------------------------------------------------------------
def test_coast_known_answer_values():
    N, icoast, ell = 200, 101, 16.0
    mask = np.ones((N, N), bool)
    mask[:, icoast - 1:] = False
    g = O.Grid(O.CART, N, N, 0.0, 1.0, 0.0, 1.0, mask=mask)
    jm = N // 2 - 1
    xs = np.arange(N, dtype=float)
    xc = np.broadcast_to(xs - xs[icoast - 1], (N, N)).copy()
    ds = (1, 4, 8, 16)
    mass, cent, wid = {}, {}, {}
    for strat in (O.ZEROFILL, O.DEFORMABLE):
        p = O.Plan(g, O.GAUSSIAN, 6.0, ell, strat)
        f1 = p.filter(np.ones((N, N)))
        fx = p.filter(xc)
        fx2 = p.filter(xc ** 2)
        i50 = 49
        sint = math.sqrt(fx2[jm, i50] / f1[jm, i50] - (fx[jm, i50] / f1[jm, i50]) ** 2)
        pts = [icoast - 1 - d for d in ds]
        mass[strat] = np.array([f1[jm, i] for i in pts])
        cent[strat] = np.array([fx[jm, i] / f1[jm, i] - xc[jm, i] for i in pts])
        wid[strat] = np.array([math.sqrt(fx2[jm, i] / f1[jm, i] - (fx[jm, i] / f1[jm, i]) ** 2) / sint for i in pts])
    np.testing.assert_allclose(cent[O.ZEROFILL], cent[O.DEFORMABLE], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(wid[O.ZEROFILL], wid[O.DEFORMABLE], rtol=1e-12)
    np.testing.assert_allclose(cent[O.ZEROFILL] / ell, [-0.211, -0.111, -0.032, 0.0], atol=5e-3)
    np.testing.assert_allclose(wid[O.ZEROFILL], [0.621, 0.747, 0.897, 0.998], atol=5e-3)
    np.testing.assert_allclose(mass[O.ZEROFILL], [0.543, 0.776, 0.948, 0.9996], atol=5e-3)
    np.testing.assert_allclose(mass[O.DEFORMABLE], 1.0, atol=1e-12)


# ---------------------------------------------------------------------------------------------
# test/test_diagnostics.jl:105-130 -- rigid rotation has Pi = 0 in the interior (Cartesian).
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("scale", [5000.0, 10000.0, 20000.0])
def test_rigid_rotation_cartesian_pi_is_zero(scale):
    n, Om = 101, 1e-4
    g = O.Grid(O.CART, n, n, -50e3, 1000.0, -50e3, 1000.0)
    x = -50e3 + 1000.0 * np.arange(n)
    X, Y = np.meshgrid(x, x)
    r = O.Plan(g, O.TOPHAT, 0.0, scale).compute_pi(-Om * Y, Om * X)
    assert np.max(np.abs(r["Pi"][39:60, 39:60])) < 1e-10


# ---------------------------------------------------------------------------------------------
# test/test_validation.jl:196-267 -- linear fields reproduce exactly; Pi = 0 for rotation and
# pure strain; the Gaussian's discrete second moment is l^2/12 (alpha=6), the disk's ~l^2/16.
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("kernel", [O.TOPHAT, O.GAUSSIAN])
def test_linear_fields_and_second_moment(kernel):
    N, dx, Om = 64, 1000.0, 1e-4
    ell = 6 * dx
    x0 = -(N // 2) * dx
    g = O.Grid(O.CART, N, N, x0, dx, x0, dx)
    p = O.Plan(g, kernel, 6.0, ell)
    xs = x0 + dx * np.arange(N)
    X, Y = np.meshgrid(xs, xs)
    pad = math.ceil(O.kernel_radius(kernel, 6.0, ell) / dx) + 1
    ii = slice(pad, N - pad)
    f1 = p.filter(np.ones((N, N)))
    fy = p.filter(Y)
    fy2 = p.filter(Y ** 2)
    s2 = fy2 / f1 - (fy / f1) ** 2
    s2i = s2[N // 2 - 1, N // 2 - 1]
    assert np.max(np.abs(s2[ii, ii] - s2i)) < 1e-12 * s2i
    if kernel == O.GAUSSIAN:
        assert s2i == pytest.approx(ell ** 2 / 12, rel=1e-9)
    else:
        assert s2i == pytest.approx(ell ** 2 / 16, rel=0.06)
    for u, v in ((-Om * Y, Om * X), (Om * Y, Om * X)):
        ub, vb = p.filter(u), p.filter(v)
        uscl = np.max(np.abs(u))
        assert np.max(np.abs(ub[ii, ii] - u[ii, ii])) < 1e-14 * uscl
        assert np.max(np.abs(vb[ii, ii] - v[ii, ii])) < 1e-14 * uscl
        Pi = p.compute_pi(u, v)["Pi"]
        assert np.max(np.abs(Pi[ii, ii])) < 1e-11 * (Om ** 3 * s2i)


# ---------------------------------------------------------------------------------------------
# test/test_grids.jl:130-179 on uniform axes -- sphere metric division of the derivatives, a
# regional edge that does not wrap, and solid-body rotation giving Pi ~ 0.
# ---------------------------------------------------------------------------------------------
def test_sphere_derivative_metric_and_regional_edge():
    lon0, dlon = 0.0, math.radians(3.0)
    lat0, dlat = math.radians(-40.0), math.radians(5.0)
    nx, ny = 31, 15
    g = O.Grid(O.SPHERE, nx, ny, lon0, dlon, lat0, dlat, R_EARTH, False, False)
    p = O.Plan(g, O.TOPHAT, 0.0, 5e5)
    lon, lat = p.coords()
    LON, LAT = np.meshgrid(lon, lat)
    dx_ = p.ddx(LON)
    dy_ = p.ddy(LAT)
    np.testing.assert_allclose(dx_[:, 1:-1], 1 / (R_EARTH * np.cos(LAT[:, 1:-1])), rtol=1e-8)
    np.testing.assert_allclose(dy_[1:-1, :], 1 / R_EARTH, rtol=1e-8)
    f2 = LON.copy()
    f2[2, nx - 1] += 1000.0
    assert p.ddx(f2)[2, 0] == pytest.approx(dx_[2, 0])


@pytest.mark.parametrize("kernel,scale", [(O.TOPHAT, 5e5), (O.GAUSSIAN, 2e5)])
def test_sphere_solid_body_rotation_pi_is_zero(kernel, scale):
    U = 5.0
    g = O.Grid(O.SPHERE, 31, 15, 0.0, math.radians(3.0), math.radians(-40.0), math.radians(5.0), R_EARTH)
    p = O.Plan(g, kernel, 4.0, scale)
    _, lat = p.coords()
    u = np.broadcast_to(U * np.cos(lat)[:, None], (15, 31)).copy()
    Pi = p.compute_pi(u, np.zeros_like(u))["Pi"]
    assert np.max(np.abs(Pi[1:-1, 1:-1])) < 1e-6


# ---------------------------------------------------------------------------------------------
# test/test_derivatives.jl:3-61 -- exact for linear fields (boundary included), 2nd-order rate.
# ---------------------------------------------------------------------------------------------
def test_ddx_exact_for_linear_fields_including_boundary():
    g = O.Grid(O.CART, 6, 6, 0.0, 2.0, 0.0, 2.0)
    p = O.Plan(g, O.TOPHAT, 0.0, 4.0)
    x = 2.0 * np.arange(6)
    f = np.broadcast_to(3.0 * x + 1.0, (6, 6)).copy()
    d = p.ddx(f)
    assert d[2, 1] == pytest.approx(3.0)
    assert d[2, 0] == pytest.approx(3.0)
    assert d[2, 5] == pytest.approx(3.0)


def test_ddx_is_second_order():
    L = 100.0
    k = 2 * math.pi / L
    errs = []
    for N in (40, 80, 160, 320):
        h = L / (N - 1)
        g = O.Grid(O.CART, N, 3, 0.0, h, 0.0, 1.0)
        p = O.Plan(g, O.TOPHAT, 0.0, 4 * h)
        x = h * np.arange(N)
        f = np.broadcast_to(np.sin(k * x), (3, N)).copy()
        d = p.ddx(f)
        errs.append(np.max(np.abs(d[:, 2:N - 2] - k * np.cos(k * x[2:N - 2]))))
    for a, b in zip(errs, errs[1:]):
        assert 1.8 < math.log2(a / b) < 2.2


# ---------------------------------------------------------------------------------------------
# test/test_validation.jl:150-190 -- filter(div u) == div(filter u) on a periodic grid, and a
# divergence-free field stays divergence-free.
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("N", [64, 96])
def test_filter_commutes_with_divergence_periodic(N):
    dx = 1000.0
    g = O.Grid(O.CART, N, N, 0.0, dx, 0.0, dx, periodic_x=True, periodic_y=True)
    u, v = spectral_field(N, dx, 3.0, symbol="stencil")
    p0 = O.Plan(g, O.TOPHAT, 0.0, 8 * dx)
    du, dv = p0.ddx(u), p0.ddy(v)
    divu = du + dv
    scl = max(np.max(np.abs(du)), np.max(np.abs(dv)))
    assert np.max(np.abs(divu)) < 1e-12 * scl
    for kern in (O.GAUSSIAN, O.TOPHAT):
        for ell in (8 * dx, 16 * dx):
            p = O.Plan(g, kern, 6.0, ell)
            ub, vb = p.filter(u), p.filter(v)
            dub, dvb = p.ddx(ub), p.ddy(vb)
            div_f = dub + dvb
            s2 = max(np.max(np.abs(dub)), np.max(np.abs(dvb)))
            assert np.max(np.abs(div_f)) < 1e-11 * s2
            assert np.max(np.abs(p.filter(divu) - div_f)) < 1e-11 * s2


# ---------------------------------------------------------------------------------------------
# test/test_validation.jl:68-144 -- the recovered filtering-spectrum slope is min(alpha, p+2).
# ---------------------------------------------------------------------------------------------
def test_filtering_spectrum_slope_saturates_at_minus_three():
    N, dx = 256, 1000.0
    g = O.Grid(O.CART, N, N, 0.0, dx, 0.0, dx, periodic_x=True, periodic_y=True)
    scales = 10 ** np.linspace(math.log10(5 * dx), math.log10(64 * dx), 17)
    kl = 1.0 / scales
    w = [i for i in range(len(scales)) if 8 * dx <= scales[i] <= 40 * dx]
    got = {}
    for kname, kern in (("Gaussian", O.GAUSSIAN), ("TopHat", O.TOPHAT)):
        for a in (5 / 3, 4.0, 7.0):
            u, v = spectral_field(N, dx, a)
            assert fourier_slope(u, v, dx, 6, 32) == pytest.approx(-a, abs=0.05)
            cum = O.cumulative_energy(g, u, v, kern, 6.0, scales)
            Et = O.spectral_density(cum, kl)
            got[(kname, a)] = logfit(kl[w], Et[w])
    for kname in ("Gaussian", "TopHat"):
        assert got[(kname, 5 / 3)] == pytest.approx(-5 / 3, abs=0.20)
        assert -3.15 < got[(kname, 7.0)] < -2.75
        assert -3.10 < got[(kname, 4.0)] < -2.60
        assert got[(kname, 7.0)] < got[(kname, 4.0)] < got[(kname, 5 / 3)]
    for a in (5 / 3, 4.0, 7.0):
        assert got[("Gaussian", a)] == pytest.approx(got[("TopHat", a)], abs=0.05)


# ---------------------------------------------------------------------------------------------
# Kernels.jl:307, 318-324, 354-359 -- radii and weights.
# ---------------------------------------------------------------------------------------------
def test_kernel_radius_and_weight():
    assert O.kernel_radius(O.TOPHAT, 0.0, 10.0) == 5.0
    assert O.kernel_radius(O.GAUSSIAN, 6.0, 1.0) == pytest.approx(math.sqrt(-math.log(1e-10) / 6.0))
    assert O.kernel_radius(O.GAUSSIAN, 4.0, 1.0) == pytest.approx(2.3993, abs=1e-4)
    assert O.kernel_weight(O.TOPHAT, 0.0, 5.0, 10.0) == 1.0
    assert O.kernel_weight(O.TOPHAT, 0.0, 5.0000001, 10.0) == 0.0
    assert O.kernel_weight(O.GAUSSIAN, 4.0, 0.5, 1.0) == pytest.approx(math.exp(-1.0))


def test_c1_footprint_statistics():
    """The 0.25-degree sphere at l = 100 km (alpha = 4): entries per latitude band."""
    d = math.radians(0.25)
    g = O.Grid(O.SPHERE, 1440, 720, d / 2, d, math.radians(-89.875), d, R_EARTH, True, False)
    di, dj, w, ptr = O.Plan(g, O.GAUSSIAN, 4.0, 1e5).footprint()
    n = np.diff(ptr)
    assert n[360] == 241 and n[0] == 12349 and n[-1] == 12349
    assert n.sum() / 720 == pytest.approx(872.9, abs=0.1)
    # each band's longitude offsets in one row are a contiguous symmetric interval
    for b in (0, 100, 360):
        lo, hi = ptr[b], ptr[b + 1]
        for r in np.unique(dj[lo:hi]):
            sel = di[lo:hi][dj[lo:hi] == r]
            assert np.all(np.diff(sel) == 1)
