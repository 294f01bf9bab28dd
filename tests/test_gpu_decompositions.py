"""tau = Leonard + Cross + Reynolds and the strain / convergence split of Pi on the GPU, checked
against the same steps composed from the oracle's filter and derivatives (the reference's own
formulas, Diagnostics.jl:1350-1527 and 1724-1852)."""
import numpy as np
import pytest

import cgef_b200 as cg
from cgef_b200 import synthetic as S
from helpers import oracle_plan, rel_l2

pytestmark = pytest.mark.gpu


def oracle_tau_parts(op, u, v, mask, sphere, grid):
    """Diagnostics.jl:1432-1461 (plane) and 1467-1525 (sphere), step for step on the oracle."""
    F = op.filter
    if not sphere:
        comps = [u, v]
    else:
        lam = grid.x.start + grid.x.step * np.arange(grid.nx)
        phi = grid.y.start + grid.y.step * np.arange(grid.ny)
        L, P = np.meshgrid(lam, phi)
        sl, cl, sp, cp = np.sin(L), np.cos(L), np.sin(P), np.cos(P)
        act = np.ones(grid.shape, bool) if mask is None else mask
        comps = [np.where(act, -sl * u - sp * cl * v, 0.0), np.where(act, cl * u - sp * sl * v, 0.0),
                 np.where(act, cp * v, 0.0)]
    nv = len(comps)
    ub = [F(c) for c in comps]
    up = [c - b for c, b in zip(comps, ub)]
    ubb = [F(b) for b in ub]
    upb = [F(p) for p in up]
    M = lambda f, g, fb, gb: F(f * g) - fb * gb
    Lp, Cp, Rp = {}, {}, {}
    for i in range(nv):
        for j in range(i, nv):
            Lp[i, j] = M(ub[i], ub[j], ubb[i], ubb[j])
            Cp[i, j] = (2.0 * M(ub[i], up[i], ubb[i], upb[i]) if i == j else
                        M(ub[i], up[j], ubb[i], upb[j]) + M(up[i], ub[j], upb[i], ubb[j]))
            Rp[i, j] = M(up[i], up[j], upb[i], upb[j])
    out = {}
    for name, T in (("L", Lp), ("C", Cp), ("R", Rp)):
        if not sphere:
            out[name] = {"xx": T[0, 0], "xy": T[0, 1], "yy": T[1, 1]}
            continue
        e = np.stack([-sl, cl, np.zeros_like(sl)])
        n = np.stack([-sp * cl, -sp * sl, cp])
        full = lambda a, b: T[min(a, b), max(a, b)]
        proj = lambda x, y: sum(x[a] * full(a, b) * y[b] for a in range(3) for b in range(3))
        act = np.ones(grid.shape, bool) if mask is None else mask
        out[name] = {"xx": np.where(act, proj(e, e), 0.0), "xy": np.where(act, proj(e, n), 0.0),
                     "yy": np.where(act, proj(n, n), 0.0)}
    return out


@pytest.mark.parametrize("geometry", ["plane", "sphere"])
def test_tau_decomposition_matches_oracle_and_sums_to_tau(geometry):
    if geometry == "plane":
        g = S.cartesian_grid(n=96)
        mask = np.ones(g.shape, bool)
        mask[30:44, 10:60] = False
        g = g.with_mask(mask)
        u, v = S.cartesian_fields(n=96, seed=5)
        kern, ell = cg.GaussianKernel(4.0), 6000.0
    else:
        g = S.sphere_grid(144, 72)
        g = g.with_mask(S.land_mask(g, seed=3))
        u, v = S.sphere_fields(g, seed=3, lmax=60)
        kern, ell = cg.GaussianKernel(4.0), 6e5
    parts = cg.tau_decomposition(u, v, g, kern, ell)
    ref = oracle_tau_parts(oracle_plan(g, kern, ell), u, v, g.mask, geometry == "sphere", g)
    for name in ("L", "C", "R"):
        for c in ("xx", "xy", "yy"):
            assert rel_l2(parts[name][c], ref[name][c]) < 1e-9, (name, c)
    # L + C + R = tau (the flux's own tau)
    f = cg.compute_Pi_fields(u, v, g, kern, ell)
    for c, k in (("xx", "tau_xx"), ("xy", "tau_xy"), ("yy", "tau_yy")):
        total = parts["L"][c] + parts["C"][c] + parts["R"][c]
        assert rel_l2(total, f[k]) < 1e-9, c


@pytest.mark.parametrize("masked", [False, True])
def test_strain_convergence_split_matches_oracle_and_pi(masked):
    g = S.cartesian_grid(n=128, periodic=(True, not masked))
    if masked:
        m = np.ones(g.shape, bool)
        m[50:70, :40] = False
        g = g.with_mask(m)
    u, v = S.cartesian_fields(n=128, seed=9)
    kern, ell = cg.GaussianKernel(4.0), 8000.0
    out = cg.compute_Pi_strain_convergence(u, v, g, kern, ell)
    op = oracle_plan(g, kern, ell)
    r = op.compute_pi(u, v)
    ux, vy = r["S_xx"], r["S_yy"]
    uy = op.ddy(r["ubar"])
    vx = op.ddx(r["vbar"])
    act = np.ones(g.shape, bool) if g.mask is None else g.mask
    txx, txy, tyy = r["tau_xx"], r["tau_xy"], r["tau_yy"]
    pa = np.where(act, (tyy - txx) * (ux - vy) / 2 - txy * (uy + vx), 0.0)
    pd = np.where(act, (tyy + txx) * (ux + vy) / 2, 0.0)
    ref = {"strain": pa, "convergence": pd, "total": pa - pd, "divergence": np.where(act, ux + vy, 0.0),
           "strain_magnitude": np.where(act, np.sqrt((ux - vy) ** 2 + (uy + vx) ** 2), 0.0)}
    for k, val in ref.items():
        assert rel_l2(out[k], val) < 1e-9, k
    # the reference's cross-check: Pi_alpha - Pi_delta is compute_Pi's Pi to round-off
    Pi = cg.compute_Pi(None, u, v, None, g, kern, ell)
    assert rel_l2(out["total"], Pi) < 1e-12


def test_strain_convergence_is_refused_on_the_sphere():
    g = S.sphere_grid(72, 36)
    u = np.zeros(g.shape)
    with pytest.raises(cg.ArgumentError):
        cg.compute_Pi_strain_convergence(u, u, g, cg.GaussianKernel(4.0), 5e5)
