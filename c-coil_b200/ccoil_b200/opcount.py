"""Algorithmic work per unit, used for roofline.achieved.

Counts are taken from the reference's CPU integrands, one per floating-point
add, subtract, multiply, divide, square root and logarithm as written there:

  fields fast  src/Coil/Fields/CalculateFieldsFast.cxx  A :63-77  B :142-154  G :225-253
  fields slow  src/Coil/Fields/CalculateFieldsSlow.cxx  A :72-76  B :149-157  G :236-250

A *coil-point evaluation* is one coil at one point at that coil's
PrecisionArguments: nodes x FLOPS_PER_NODE + thickness(/length) nodes x
PER_T_FLOPS + PER_POINT_FLOPS (transform into the coil frame, cylindrical
coordinates, rotation of the result back).
"""
import numpy as np

# field index: 0 = A (E), 1 = B, 3 = G
FLOPS_PER_NODE = {
    (0, True): 22, (1, True): 24, (3, True): 62,   # fast method (RECTANGULAR, THIN)
    (0, False): 9, (1, False): 14, (3, False): 38,  # slow method (FLAT, FILAMENT)
}
PER_T_FLOPS = {0: 6, 1: 9, 3: 12}
PER_POINT_FLOPS = {0: 40, 1: 40, 3: 90}


def nodes_of(prec, fast):
    """(angular nodes, thickness(-length) node pairs) of a PrecisionArguments tuple; the
    fast method integrates the length analytically, so its length layer is not evaluated."""
    aB, tB, lB, aI, tI, lI = prec
    return aB * aI, tB * tI * (1 if fast else lB * lI)


def coil_point_flops(field, prec, fast):
    f = 0 if field == 2 else field
    nphi, ntl = nodes_of(prec, fast)
    return nphi * ntl * FLOPS_PER_NODE[(f, bool(fast))] + ntl * PER_T_FLOPS[f] + PER_POINT_FLOPS[f]


def group_flops_per_point(field, coils):
    """Sum over coils of the flops of one coil-point evaluation (coils: Coil objects)."""
    return float(sum(coil_point_flops(field, c.struct().precision.as_tuple(), c.is_using_fast_method())
                     for c in coils))


def group_nodes_per_point(coils):
    total = 0
    for c in coils:
        nphi, ntl = nodes_of(c.struct().precision.as_tuple(), c.is_using_fast_method())
        total += nphi * ntl
    return float(total)


def summary(coils):
    return {"coils": len(coils), "nodes_per_point": group_nodes_per_point(coils),
            "flops_per_point": {k: group_flops_per_point(f, coils) for k, f in (("A", 0), ("B", 1), ("G", 3))}}


__all__ = ["FLOPS_PER_NODE", "PER_T_FLOPS", "PER_POINT_FLOPS", "coil_point_flops", "group_flops_per_point",
           "group_nodes_per_point", "summary", "np"]
