"""The C ABI loads and exports every symbol include/n4b200.h declares, and
its host-side logic (defaults, sizes, validation) works without a GPU."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "n4b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(n4_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("n4_run", "n4_run_host", "n4_run_batched", "n4_fit_bspline3d", "n4_evaluate_bspline3d",
              "n4_upsample_lattice3d", "n4_sharpen_image", "n4_convergence", "n4_create", "n4_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import n4b200
    from n4b200 import _lib
    lib = n4b200.library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    # and the binding declares exactly those
    assert sorted(n for n, _, _ in _lib.SIGNATURES) == declared_functions()


def test_struct_layouts_match_header():
    from n4b200 import _lib
    # n4_params_t: 7 x 4 B + 8 x 4 B + 6 x 4 B
    assert C.sizeof(_lib.n4_params_t) == 4 * (7 + 8 + 6)
    assert C.sizeof(_lib.n4_report_t) == 4 * 2 + 4 * 8 * 2 + 4 * 3 + 4 + 8 + 4 * 2 + 8 * 2 + 4 * 2
    assert _lib.n4_report_t.device_begin_ns.offset % 8 == 0
    T = _lib.N4_TUNE_MAX
    assert C.sizeof(_lib.n4_tune_report_t) == 4 + 4 * T * 3 + 4 + 4 + 4 * T * 3 + 4 + 4 + 4 * T * 3 + 4 + 4 * T
    assert C.sizeof(_lib.n4_component_tune_t) == 4 + 4 * T * 4 + 8 + 4 + 4 * T * 3 + 8
    assert C.sizeof(_lib.n4_timings_t) == 4 * 4 + 4 + 4 + 8 + 8 + 4 * 6


def test_defaults_match_reference_n4param():
    """Defaults of N4Param (cudaN4.h:24-94)."""
    import n4b200
    p = n4b200.N4Param()
    assert p.NumberOfHistogramBins == 200
    assert p.WienerFilterNoise == pytest.approx(0.01)
    assert p.BiasFieldFullWidthAtHalfMaximum == pytest.approx(0.15)
    assert (p.NumberOfControlPoints_x, p.NumberOfControlPoints_y, p.NumberOfControlPoints_z) == (4, 4, 4)
    assert p.NumberOfFittingLevels == 4
    assert p.MaximumNumberOfIterations == 50
    assert p.ConvergenceThreshold == pytest.approx(0.001)
    assert p.low_value == pytest.approx(10.0)
    assert p.SplineOrder == 3 and p.ShrinkFactor == 1


def test_lattice_dims():
    """(2^(L-1)(ncpt-3)+3) per axis, cudaN4.h:359 / main.cpp:87-91."""
    import n4b200
    assert n4b200.lattice_dims(n4b200.N4Param()) == (11, 11, 11)
    p = n4b200.N4Param(NumberOfFittingLevels=3, NumberOfControlPoints_x=5)
    assert n4b200.lattice_dims(p) == (11, 7, 7)


def test_validation_without_a_gpu():
    import n4b200
    from n4b200 import N4Error
    with pytest.raises(N4Error, match="UNSUPPORTED_SPLINE_ORDER"):
        n4b200.lattice_dims(n4b200.N4Param(SplineOrder=2))
    with pytest.raises(N4Error, match="INVALID_ARG"):
        n4b200.lattice_dims(n4b200.N4Param(NumberOfHistogramBins=1))
    with pytest.raises(N4Error, match="INVALID_ARG"):
        n4b200.lattice_dims(n4b200.N4Param(NumberOfControlPoints=3))
    with pytest.raises(N4Error, match="TOO_LARGE"):
        n4b200.lattice_dims(n4b200.N4Param(NumberOfFittingLevels=8))
    with pytest.raises(AttributeError):
        n4b200.N4Param(NotAField=1)


def test_volume_size_checks_without_a_gpu():
    """The size checks of a run (shrink divisibility, voxel and row limits)
    happen on the host before any device work."""
    import n4b200
    from n4b200 import N4Error
    p = n4b200.N4Param(ShrinkFactor=4)
    assert n4b200.fitting_dims(p, (256, 256, 176)) == (64, 64, 44)
    assert n4b200.fitting_dims(n4b200.N4Param(ShrinkFactor=2), (512, 512, 320)) == (256, 256, 160)
    with pytest.raises(N4Error, match="INVALID_ARG"):
        n4b200.fitting_dims(p, (256, 256, 174))          # not a multiple of the shrink factor
    with pytest.raises(N4Error, match="INVALID_ARG"):
        n4b200.fitting_dims(p, (0, 256, 176))
    # 65536 x 65536 x 8 (2^35 voxels, 34 GB): fewer than 2^40 voxels, but
    # 2^32 rows, which the full-resolution correction cannot index
    with pytest.raises(N4Error, match="TOO_LARGE"):
        n4b200.fitting_dims(p, (65536, 65536, 8))
    assert n4b200.fitting_dims(p, (65532, 65536, 8)) == (16383, 16384, 2)
    with pytest.raises(N4Error, match="TOO_LARGE"):
        n4b200.fitting_dims(n4b200.N4Param(ShrinkFactor=1), (64, 64, 2048))   # fitting rows > 1024


def test_fit_size_checks_precede_device_work():
    """Both standalone fits reject extents of 2^31 or more, more than 2^36
    field voxels and more than 4096 control points along an axis before any
    CUDA call (the pointers below are never dereferenced)."""
    import n4b200
    from n4b200 import _lib
    lib = n4b200.library()
    fake = C.c_void_p(256)
    cases = [((4, 4, 4), (1 << 31, 1, 1)),          # extent above INT_MAX
             ((4, 4, 4), (1 << 20, 1 << 16, 1)),    # 2^36 voxels
             ((4, 4, 5000), (64, 64, 64))]          # control points per axis
    for nc, dims in cases:
        st = lib.n4_fit_bspline3d_noalloc(fake, None, *nc, *dims, 1e-3, 0, fake, None)
        assert _lib.STATUS[st] == "N4_ERR_TOO_LARGE", (nc, dims)
        # the allocating fit checks sizes before it touches its (here fake) context
        st = lib.n4_fit_bspline3d(fake, fake, None, *nc, *dims, 1e-3, 0, fake, None)
        assert _lib.STATUS[st] == "N4_ERR_TOO_LARGE", (nc, dims)


def test_status_strings():
    import n4b200
    lib = n4b200.library()
    assert lib.n4_status_string(3) == b"empty mask"
    assert lib.n4_version().startswith(b"n4b200")


def test_create_reports_missing_device():
    """n4_create returns a status instead of crashing when no GPU is visible."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import n4b200
    lib = n4b200.library()
    h = C.c_void_p()
    assert lib.n4_create(C.byref(h), 0) == 9   # N4_ERR_NO_DEVICE
    assert lib.n4_destroy(None) == 0


def test_python_flags_match_the_header():
    """Every N4_FLAG_* constant of the Python binding has the header's value
    (the parametrised ones for every argument)."""
    from n4b200 import _lib
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    consts = dict(re.findall(r"#define\s+N4_FLAG_([A-Z0-9_]+)\s+(0x[0-9a-fA-F]+)u", src))
    assert consts, "no flag constants found"
    for name, value in consts.items():
        assert getattr(_lib, "FLAG_" + name) == int(value, 16), name
    pattern = r"#define\s+N4_FLAG_([A-Z0-9_]+)\(k\)\s+\(\(\(unsigned int\)\(k\) & (\d+)u\) << (\d+)\)"
    shifts = {name: (int(mask), int(shift)) for name, mask, shift in re.findall(pattern, src)}
    assert "SUB_BATCHES" in shifts and "CLUSTER_SIZE" in shifts
    import n4b200
    for k in range(8):
        assert _lib.FLAG_SUB_BATCHES(k) == (k & shifts["SUB_BATCHES"][0]) << shifts["SUB_BATCHES"][1]
    for k in range(17):
        assert n4b200.cluster_size_flag(k) == (k & shifts["CLUSTER_SIZE"][0]) << shifts["CLUSTER_SIZE"][1]
