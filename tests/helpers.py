"""Test helpers: the same grid for the CUDA library and for the oracle, and error metrics."""
import numpy as np

import cgef_b200 as cg
import oracle as O


def oracle_grid(g: "cg.StructuredGrid", mask=None) -> O.Grid:
    m = g.mask if mask is None else mask
    return O.Grid(O.SPHERE if g.is_spherical else O.CART, g.nx, g.ny, g.x.start, g.x.step, g.y.start, g.y.step,
                  g.geometry.R if g.is_spherical else 6.371e6, g.periodic[0], g.periodic[1], m)


def oracle_plan(g, kernel, scale, strategy=None, engine=O.ENGINE_AUTO, mask=None):
    st = O.DEFORMABLE if isinstance(strategy, cg.Deformable) else O.ZEROFILL
    k = O.TOPHAT if isinstance(kernel, cg.TopHatKernel) else O.GAUSSIAN
    return O.Plan(oracle_grid(g, mask), k, float(getattr(kernel, "alpha", 0.0)), float(scale), st, engine)


def rel_l2(x, ref, sel=None):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if sel is not None:
        x, ref = x[sel], ref[sel]
    den = np.linalg.norm(ref)
    return np.linalg.norm(x - ref) / (den if den > 0 else 1.0)


def max_rel(x, ref):
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.max(np.abs(ref))
    return np.max(np.abs(x - ref)) / (scale if scale > 0 else 1.0)
