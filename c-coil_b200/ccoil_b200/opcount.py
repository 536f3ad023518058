"""Algorithmic work per unit and the pipe model used for roofline.achieved.

A *coil-point evaluation* is one coil at one point at that coil's
PrecisionArguments.  Its work is nodes x (work per node) plus small per
thickness(/length)-node and per-point terms.

FP64 kernel.  The per-node operation mix is that of the reference's CPU
integrands, whose operation sequence the FP64 kernel follows one for one
(add/subtract/multiply, divide, square root, logarithm):

  fields fast  src/Coil/Fields/CalculateFieldsFast.cxx  A :63-77  B :142-154  G :225-253
  fields slow  src/Coil/Fields/CalculateFieldsSlow.cxx  A :72-76  B :149-157  G :236-250

Add, subtract and multiply each take one FP64-pipe instruction slot; a divide,
square root or logarithm takes rate(FMA) / rate(op) slots, with the rates
measured on the device by ccoil_measure_op_rates.

The FP32-compensated kernels do more arithmetic per node than the reference's
integrand (closed-form mirror differences, compensated sums); their roofline
counts the same algorithmic flops, and ncu's pipe utilisation (committed under
profiles/) describes the kernels themselves.
"""

# field index: 0 = A (E), 1 = B, 3 = G; (field, fast method) ->
# (add/sub/mul, div, sqrt, log) per node of the reference integrand
OPS_PER_NODE_64 = {
    (0, True): (13, 2, 3, 1), (0, False): (5, 1, 1, 0),
    (1, True): (17, 3, 2, 0), (1, False): (11, 1, 1, 0),
    (3, True): (53, 6, 2, 0), (3, False): (33, 2, 1, 0),
}
# algorithmic flops per node: every operation of the reference integrand counts one
FLOPS_PER_NODE = {k: sum(v) for k, v in OPS_PER_NODE_64.items()}
PER_T_FLOPS = {0: 6, 1: 9, 3: 12}
PER_POINT_FLOPS = {0: 40, 1: 40, 3: 90}


def nodes_of(prec, fast):
    """(angular nodes, thickness(-length) node pairs) of a PrecisionArguments tuple; the
    fast method integrates the length analytically, so its length layer is not evaluated."""
    aB, tB, lB, aI, tI, lI = prec
    return aB * aI, tB * tI * (1 if fast else lB * lI)


def _field(field):
    return 0 if field == 2 else field


def coil_point_flops(field, prec, fast):
    f = _field(field)
    nphi, ntl = nodes_of(prec, fast)
    return nphi * ntl * FLOPS_PER_NODE[(f, bool(fast))] + ntl * PER_T_FLOPS[f] + PER_POINT_FLOPS[f]


def _coils(coils):
    for c in coils:
        yield c.struct().precision.as_tuple(), bool(c.is_using_fast_method())


def group_flops_per_point(field, coils):
    """Sum over coils of the flops of one coil-point evaluation (coils: Coil objects)."""
    return float(sum(coil_point_flops(field, p, fast) for p, fast in _coils(coils)))


def group_nodes_per_point(coils):
    total = 0
    for p, fast in _coils(coils):
        nphi, ntl = nodes_of(p, fast)
        total += nphi * ntl
    return float(total)


def fp64_slots_per_point(field, coils, rates):
    """FP64-pipe instruction slots per point for the group: rates = ccoil_measure_op_rates."""
    f = _field(field)
    c_div, c_sqrt, c_log = (rates[0] / rates[k] for k in (1, 2, 3))
    total = 0.0
    for p, fast in _coils(coils):
        nphi, ntl = nodes_of(p, fast)
        am, dv, sq, lg = OPS_PER_NODE_64[(f, fast)]
        total += nphi * ntl * (am + dv * c_div + sq * c_sqrt + lg * c_log) + ntl * PER_T_FLOPS[f] \
            + PER_POINT_FLOPS[f]
    return total


def summary(coils):
    return {"coils": len(coils), "nodes_per_point": group_nodes_per_point(coils),
            "flops_per_point": {k: group_flops_per_point(f, coils) for k, f in (("A", 0), ("B", 1), ("G", 3))}}


__all__ = ["OPS_PER_NODE_64", "FLOPS_PER_NODE", "PER_T_FLOPS", "PER_POINT_FLOPS",
           "nodes_of", "coil_point_flops", "group_flops_per_point", "group_nodes_per_point",
           "fp64_slots_per_point", "summary"]
