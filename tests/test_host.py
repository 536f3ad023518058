"""Host-side logic of the product (no GPU needed): precision balancing, coil set-up,
Gauss-Legendre tables, the exported C-ABI, and argument checking."""
import ctypes

import numpy as np
import pytest

from conftest import HAS_GPU, header_functions


def test_library_exports_every_header_symbol(ccoil):
    names = header_functions()
    assert "ccoil_compute_fields" in names and len(names) >= 10
    lib = ccoil.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


# The reference's GPU entry points (include/ccoil_reference_abi.h) with their C++
# names, as g++ mangles them for the TYPE=double structs
REFERENCE_ENTRY_SYMBOLS = [
    "_Z32Calculate_hardware_accelerated_ax8CoilDataPK10VectorDataPS0_",
    "_Z32Calculate_hardware_accelerated_bx8CoilDataPK10VectorDataPS0_",
    "_Z32Calculate_hardware_accelerated_gx8CoilDataPK10VectorDataP10MatrixData",
    "_Z42Calculate_mutual_inductance_configurationsxxPK21CoilPairArgumentsDataPK20CoilPairPositionDataPd",
    "_Z41Calculate_force_and_torque_configurationsxxPK21CoilPairArgumentsDataPK20CoilPairPositionDataP15ForceTorqueData",
    "_Z38Calculate_hardware_accelerated_a_groupxxPK8CoilDataPK10VectorDataPS2_",
    "_Z38Calculate_hardware_accelerated_b_groupxxPK8CoilDataPK10VectorDataPS2_",
    "_Z38Calculate_hardware_accelerated_e_groupxxPK8CoilDataPK10VectorDataPS2_",
    "_Z38Calculate_hardware_accelerated_g_groupxxPK8CoilDataPK10VectorDataP10MatrixData",
    "_Z48Calculate_mutual_inductance_configurations_groupxxx17SecondaryCoilDataPK8CoilDataPK25SecondaryCoilPositionDataPd",
    "_Z47Calculate_force_and_torque_configurations_groupxxx17SecondaryCoilDataPK8CoilDataPK25SecondaryCoilPositionDataP15ForceTorqueData",
]


def test_library_exports_the_reference_entry_points(ccoil):
    lib = ccoil.lib()
    missing = [n for n in REFERENCE_ENTRY_SYMBOLS if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_gpu_glue_links_against_the_library(ccoil):
    """The reference's unmodified GPU glue (built with USE_GPU, oracle/Makefile target
    ref-gpu, linked with --no-undefined) loads with this library standing in for its
    CUDA kernels."""
    from oracle import Reference, REF_GPU_SO
    if not Reference.available(REF_GPU_SO):
        pytest.skip("oracle/_ref/libccoil_ref_gpu.so not built (needs the reference sources)")
    ccoil.lib()
    glue = Reference(REF_GPU_SO)
    assert hasattr(glue.lib, "ref_group_fields_dispatch")


def test_abi_version(ccoil):
    assert ccoil.lib().ccoil_abi_version() == 1


def test_precision_arguments_match_reference(ccoil, golden):
    from oracle import coil_row  # noqa: F401  (rows share the oracle's layout)
    for c, pf, cpu, gpu in zip(golden["prec_coils"], golden["prec_pf"], golden["prec_cpu"], golden["prec_gpu"]):
        coil = ccoil.Coil(c[0], c[1], c[2], int(c[3]))
        got = ccoil.PrecisionArguments.get_coil_precision_arguments_CPU(coil, pf).as_tuple()
        assert got == tuple(cpu)
        got = ccoil.PrecisionArguments.get_coil_precision_arguments_GPU(coil, pf, 80).as_tuple()
        assert got == tuple(gpu)


def test_pair_arguments_match_reference(ccoil, golden):
    for p, s, pf, cpu, gpu in zip(golden["pprec_prim"], golden["pprec_sec"], golden["pprec_pf"],
                                  golden["pprec_cpu"], golden["pprec_gpu"]):
        prim = ccoil.Coil(p[0], p[1], p[2], int(p[3]))
        sec = ccoil.Coil(s[0], s[1], s[2], int(s[3]))
        a = ccoil.CoilPairArguments.get_appropriate_coil_pair_arguments(prim, sec, pf, ccoil.ComputeMethod.CPU_ST)
        assert a.primary_precision.as_tuple() + a.secondary_precision.as_tuple() == tuple(cpu)
        a = ccoil.CoilPairArguments.get_appropriate_coil_pair_arguments(prim, sec, pf, ccoil.ComputeMethod.GPU,
                                                                        pure_gpu=True, gpu_increments=80)
        assert a.primary_precision.as_tuple() + a.secondary_precision.as_tuple() == tuple(gpu)


def test_coil_attributes_match_oracle(ccoil, oracle):
    rng = np.random.default_rng(3)
    for _ in range(50):
        R = rng.uniform(0.01, 0.5)
        a = 0.0 if rng.uniform() < 0.3 else rng.uniform(0, 0.2)
        b = 0.0 if rng.uniform() < 0.3 else rng.uniform(0, 0.2)
        pos = rng.uniform(-1, 1, 3)
        ya, za = rng.uniform(0, np.pi), rng.uniform(0, 2 * np.pi)
        c = ccoil.Coil(R, a, b, 123, 2.5, 60.0, 5.0, 8, pos, ya, za)
        info = oracle.coil_info(np.array([R, a, b, 123, 2.5, 60.0, *pos, ya, za]))
        assert c.get_thickness() == info[0] and c.get_length() == info[1]
        assert c.get_current_density() == info[2]
        assert int(c.is_using_fast_method()) == int(info[4]) and int(c.get_coil_type()) == int(info[5])
        assert np.array_equal(c.get_transformation_matrix().ravel(), info[6:15])
        assert np.array_equal(c.get_inverse_transformation_matrix().ravel(), info[15:24])


def test_legendre_tables_match_oracle(ccoil, oracle):
    for n in range(1, 101):
        x, w = ccoil.legendre(n)
        xo, wo = oracle.legendre(n)
        assert np.array_equal(x, xo) and np.array_equal(w, wo)
        assert np.all(np.diff(x) > 0) and abs(w.sum() - 2.0) < 1e-13


def test_legendre_tables_match_reference(ccoil, reference):
    for n in range(1, 101):
        x, w = ccoil.legendre(n)
        xr, wr = reference.legendre(n)
        assert np.max(np.abs(x - xr)) <= 4.5e-16
        assert np.max(np.abs(w - wr) / wr) <= 1e-15


def test_invalid_arguments_are_rejected_before_any_device_work(ccoil):
    L = ccoil.lib()
    coil = ccoil.Coil(0.1, 0.1, 0.1, 100)
    s = coil.struct()
    arr = (ccoil._lib.CoilStruct * 1)(s)
    h = ctypes.c_void_p()
    # unknown field / precision
    assert L.ccoil_field_plan_create(arr, 1, 7, 0, ctypes.byref(h)) == 1
    assert L.ccoil_field_plan_create(arr, 1, 1, 9, ctypes.byref(h)) == 1
    # negative counts / null pointers
    assert L.ccoil_field_plan_create(arr, -1, 1, 0, ctypes.byref(h)) == 1
    assert L.ccoil_compute_fields(None, 1, None, 10, 1, 0, None, 0, None) == 1
    # precision arguments out of range
    bad = ccoil._lib.CoilStruct()
    ctypes.pointer(bad)[0] = s
    bad.precision.angular_increments = 101
    arr2 = (ccoil._lib.CoilStruct * 1)(bad)
    assert L.ccoil_field_plan_create(arr2, 1, 1, 0, ctypes.byref(h)) == 1
    assert b"precision" in L.ccoil_last_error_message()
    assert L.ccoil_legendre(0, None, None) == 1
    with pytest.raises(ccoil.CCoilError):
        ccoil.legendre(101)
    # the FP64 diagnostics (logarithm, reciprocal square root, division): negative
    # count, null buffers; an empty call is a no-op
    assert L.ccoil_eval_log64(None, None, -1, None) == 1
    assert L.ccoil_eval_log64(None, None, 4, None) == 1
    assert L.ccoil_eval_log64(None, None, 0, None) == 0
    assert L.ccoil_eval_fp64_op(0, None, None, None, 4, None) == 1
    assert L.ccoil_eval_fp64_op(2, None, None, None, -1, None) == 1
    assert L.ccoil_eval_fp64_op(4, None, None, None, 0, None) == 1
    assert L.ccoil_eval_fp64_op(3, None, None, None, 0, None) == 0


def test_cpu_compute_methods_are_not_provided(ccoil):
    c = ccoil.Coil(0.1, 0.1, 0.1, 100)
    with pytest.raises(NotImplementedError):
        c.compute_all_B_field_vectors(np.zeros((2, 3)), ccoil.ComputeMethod.CPU_ST)


@pytest.mark.skipif(HAS_GPU, reason="checks the behaviour without a CUDA device")
def test_no_device_fails_loudly(ccoil):
    c = ccoil.Coil(0.1, 0.1, 0.1, 100)
    with pytest.raises(ccoil.CCoilError) as ei:
        c.compute_all_B_field_vectors(np.zeros((4, 3)))
    assert ei.value.status in (2, 6)


def test_segment_split_for_large_angular_tables(ccoil):
    # PrecisionFactor 12 on a filament: thousands of angular nodes over many blocks,
    # more than one staging segment; plan creation must accept it (host only).
    c = ccoil.Coil(0.1, 0.0, 0.0, 10, precision_factor=12.0)
    p = c.default_precision_CPU
    assert p.angular_blocks > 100
    if not HAS_GPU:
        with pytest.raises(ccoil.CCoilError):
            ccoil.FieldPlan([c.struct()], 1)


def test_negative_counts_are_rejected_without_a_device(ccoil):
    """Argument checks come before any CUDA call."""
    L = ccoil.lib()
    from ccoil_b200 import _lib
    s = _lib.CoilStruct()
    pos = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    assert L.ccoil_coil_init(0.1, 0.05, 0.1, 100, 1.0, 0.0, pos, 0.0, 0.0, 5.0, 0, ctypes.byref(s)) == 0
    arr = (_lib.CoilStruct * 1)(s)
    buf = (ctypes.c_double * 3)()
    assert L.ccoil_compute_fields(arr, 1, buf, -1, 1, 0, buf, 0, None) == 1
    assert L.ccoil_compute_fields(arr, -1, buf, 1, 1, 0, buf, 0, None) == 1
    assert L.ccoil_compute_fields(arr, 1, buf, 1, 7, 0, buf, 0, None) == 1
    assert L.ccoil_inject_allocation_failures(-1) == 1
    assert L.ccoil_check_bounded_wait(-5, None) == 1
