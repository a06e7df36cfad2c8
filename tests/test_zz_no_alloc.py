"""``n4_fit_bspline3d_noalloc`` against ``n4_fit_bspline3d``.

The no-allocation entry point runs the same fit kernels over a fixed device
scratch array instead of context workspaces, so every call must reproduce the
allocating entry point's lattice bit for bit, also when calls of different
sizes follow one another on the same scratch.  Named to be collected last, so
that it runs after the rest of the suite as well as alone.
"""
import ctypes as C

import numpy as np
import pytest

SCRATCH_BYTES = 8 << 20


def _lib():
    from n4b200 import _lib
    return _lib


def test_oversize_is_rejected_before_any_device_work():
    """The size check precedes every CUDA call, so it needs no GPU."""
    L = _lib()
    lib = L.load()
    # 1024 x 1024 rows x 16 control points along z: 128 MiB of row sums
    st = lib.n4_fit_bspline3d_noalloc(C.c_void_p(256), None, 4, 4, 16, 1024, 1024, 64, 1e-3, 0,
                                      C.c_void_p(256), None)
    assert L.STATUS[st] == "N4_ERR_TOO_LARGE"
    msg = lib.n4_last_error_string().decode()
    assert str(SCRATCH_BYTES) in msg and "n4_fit_bspline3d" in msg


def _noalloc(cuda, field, mask, nc, eps=1e-3, zero_den=False):
    L = _lib()
    out = cuda.empty(nc, dtype=cuda.float32, device=field.device)
    X, Y, Z = field.shape
    st = L.load().n4_fit_bspline3d_noalloc(field.data_ptr(), None if mask is None else mask.data_ptr(), *nc,
                                           X, Y, Z, float(eps), int(zero_den), out.data_ptr(),
                                           cuda.cuda.current_stream(field.device).cuda_stream)
    L.check(st)
    return out


@pytest.mark.gpu
def test_matches_allocating_fit_on_consecutive_calls(cuda):
    import n4b200
    rng = np.random.default_rng(31)
    cases = [((64, 64, 44), (11, 11, 11), True, False),
             ((96, 80, 60), (7, 5, 9), True, True),
             ((40, 48, 36), (4, 6, 5), False, False)]
    inputs = []
    for shape, nc, with_mask, zero_den in cases:
        f = cuda.tensor(rng.normal(0.0, 0.3, size=shape).astype(np.float32), device="cuda")
        m = cuda.tensor((rng.random(shape) < 0.7).astype(np.float32), device="cuda") if with_mask else None
        inputs.append((f, m, nc, zero_den))
    # two rounds over all cases: every call follows a call of another size
    for _ in range(2):
        for f, m, nc, zero_den in inputs:
            got = _noalloc(cuda, f, m, nc, zero_den=zero_den)
            ref = n4b200.FitBspline3D(f, m, nc, zero_den=zero_den)
            cuda.cuda.synchronize()
            assert cuda.isfinite(got).all()
            assert cuda.equal(got, ref), nc


@pytest.mark.gpu
def test_largest_fit_the_scratch_holds(cuda):
    """256 x 256 rows with 11 control points along z (the 512x512x320
    workload's fitting grid at shrink 2) fits in the fixed scratch."""
    import n4b200
    rng = np.random.default_rng(32)
    shape, nc = (256, 256, 160), (11, 11, 11)
    f = cuda.tensor(rng.normal(0.0, 0.3, size=shape).astype(np.float32), device="cuda")
    m = cuda.tensor((rng.random(shape) < 0.5).astype(np.float32), device="cuda")
    for _ in range(2):
        got = _noalloc(cuda, f, m, nc)
        ref = n4b200.FitBspline3D(f, m, nc)
        cuda.cuda.synchronize()
        assert cuda.equal(got, ref)


@pytest.mark.gpu
def test_calls_after_the_first_reserve_no_device_memory(cuda):
    """The point of the entry point: once the library's device code is loaded
    (the first call of each kernel variant may load it, and with it the fixed
    scratch array), further calls of any size leave the device's free memory
    unchanged.  Inputs and outputs are allocated before the first sample."""
    rng = np.random.default_rng(33)
    cases = [((64, 64, 44), (11, 11, 11), True), ((96, 80, 60), (7, 5, 9), False), ((40, 48, 36), (4, 6, 5), True)]
    bufs = []
    for shape, nc, with_mask in cases:
        f = cuda.tensor(rng.normal(0.0, 0.3, size=shape).astype(np.float32), device="cuda")
        m = cuda.tensor((rng.random(shape) < 0.7).astype(np.float32), device="cuda") if with_mask else None
        out = cuda.empty(nc, dtype=cuda.float32, device="cuda")
        bufs.append((f, m, nc, out))
    L = _lib()
    lib = L.load()

    def call(f, m, nc, out):
        X, Y, Z = f.shape
        L.check(lib.n4_fit_bspline3d_noalloc(f.data_ptr(), None if m is None else m.data_ptr(), *nc, X, Y, Z,
                                             1e-3, 0, out.data_ptr(),
                                             cuda.cuda.current_stream(f.device).cuda_stream))

    for b in bufs:            # warm-up: every kernel variant the later calls use
        call(*b)
    cuda.cuda.synchronize()
    free0, _ = cuda.cuda.mem_get_info()
    firsts = [b[3].clone() for b in bufs]
    for _ in range(3):
        for b in bufs:
            call(*b)
    cuda.cuda.synchronize()
    free1, _ = cuda.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    for b, first in zip(bufs, firsts):
        assert cuda.equal(b[3], first)
