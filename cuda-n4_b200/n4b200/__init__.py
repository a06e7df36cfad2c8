"""n4b200: N4 bias-field correction on NVIDIA B200, drop-in for the reference
CUDA-N4 interface.

The functions mirror the reference entry points (``cudaN4.h``) and its
numpy twin (``N4.py``) by name and argument meaning:

=================================  ==========================================
here                               reference
=================================  ==========================================
``N4Param``                        ``struct N4Param`` (cudaN4.h:24-94)
``N4``                             ``N4()`` / ``testN4()`` (cudaN4.h:343-387),
                                   ``N4()`` (N4.py:276-332)
``N4Batch``                        (new) many volumes in one launch
``FitBspline3D``                   ``FitBspline3D`` (cudaN4.h:313, N4.py:186)
``EvaluateBspline3D``              ``EvaluateBspline3D`` (cudaN4.h:288, N4.py:241)
``UpsampleLattice3D``              ``upsampleLattice3D_gpu`` (cudaN4.h:269), N4.py:132
``sharpenImage``                   ``sharpenImage`` (cudaN4.h:198, N4.py:9)
``CalculateConvergenceMeasurement````calculateConvergenceMeasurement`` (cudaN4.h:249),
                                   N4.py:121
=================================  ==========================================

Every call goes through ``libn4b200.so`` (hand-written sm_100a kernels); there
is no CPU fallback.  Inputs may be CUDA tensors (device path, outputs are
CUDA tensors) or numpy arrays (host path, outputs are numpy arrays).
Volumes are float32 ``[fx][fy][fz]`` with the last axis fastest.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import N4Error, check, n4_params_t, n4_report_t, n4_volume_t

__all__ = [
    "N4Param", "N4", "N4Batch", "N4BatchGraph", "N4Result", "Context", "FitBspline3D",
    "EvaluateBspline3D", "UpsampleLattice3D", "upsampleLattice3D", "sharpenImage",
    "CalculateConvergenceMeasurement", "calculateConvergenceMeasurement", "N4Error",
    "lattice_dims", "library", "autotune", "autotune_components", "cluster_size_flag", "warm_inputs", "N4BatchHost",
]


def library():
    """The loaded ``libn4b200.so`` (raises ImportError when it is not built)."""
    return _lib.load()


# ---------------------------------------------------------------- parameters
class N4Param:
    """Parameters of N4, with the field names of the reference's ``N4Param``.

    Defaults are the reference's (``cudaN4.h:24-94``), including
    ``low_value = 10``; synthetic phantoms with intensities around 1 need
    ``low_value = 0``.  ``MaximumNumberOfIterations`` is one count for every
    level (the CUDA reference) or a list with one count per level (N4.py).
    """

    _FIELDS = ("NumberOfHistogramBins", "WienerFilterNoise", "BiasFieldFullWidthAtHalfMaximum",
               "NumberOfControlPoints_x", "NumberOfControlPoints_y", "NumberOfControlPoints_z",
               "NumberOfFittingLevels", "MaximumNumberOfIterations", "ConvergenceThreshold",
               "low_value", "ShrinkFactor", "SplineOrder", "FitEpsilon", "flags")

    def __init__(self, **kw):
        c = n4_params_t()
        _lib.load().n4_params_default(C.byref(c))
        self.NumberOfHistogramBins = c.NumberOfHistogramBins
        self.WienerFilterNoise = c.WienerFilterNoise
        self.BiasFieldFullWidthAtHalfMaximum = c.BiasFieldFullWidthAtHalfMaximum
        self.NumberOfControlPoints_x = c.NumberOfControlPoints_x
        self.NumberOfControlPoints_y = c.NumberOfControlPoints_y
        self.NumberOfControlPoints_z = c.NumberOfControlPoints_z
        self.NumberOfFittingLevels = c.NumberOfFittingLevels
        self.MaximumNumberOfIterations = c.MaximumNumberOfIterations[0]
        self.ConvergenceThreshold = c.ConvergenceThreshold
        self.low_value = c.low_value
        self.ShrinkFactor = c.ShrinkFactor
        self.SplineOrder = c.SplineOrder
        self.FitEpsilon = c.FitEpsilon
        self.flags = c.flags
        for k, v in kw.items():
            setattr(self, k, v)

    def __setattr__(self, k, v):
        if k == "NumberOfControlPoints":
            for a in ("x", "y", "z"):
                object.__setattr__(self, f"NumberOfControlPoints_{a}", int(v))
            return
        if k not in self._FIELDS:
            raise AttributeError(f"N4Param has no field {k!r}")
        object.__setattr__(self, k, v)

    def to_c(self) -> n4_params_t:
        c = n4_params_t()
        for k in self._FIELDS:
            if k == "MaximumNumberOfIterations":
                it = self.MaximumNumberOfIterations
                its = [int(it)] * _lib.N4_MAX_LEVELS if np.isscalar(it) else list(it)
                if len(its) < self.NumberOfFittingLevels:
                    raise ValueError("one iteration count per fitting level is required")
                its = (its + [0] * _lib.N4_MAX_LEVELS)[:_lib.N4_MAX_LEVELS]
                c.MaximumNumberOfIterations[:] = [int(i) for i in its]
            else:
                setattr(c, k, getattr(self, k))
        return c

    def lattice_dims(self):
        return lattice_dims(self)

    def __repr__(self):
        return "N4Param(" + ", ".join(f"{k}={getattr(self, k)!r}" for k in self._FIELDS) + ")"


def lattice_dims(param: N4Param):
    """Control points per axis at the last level (``cudaN4.h:359``)."""
    dims = (C.c_uint * 3)()
    n = C.c_size_t()
    c = param.to_c()
    check(_lib.load().n4_lattice_dims(C.byref(c), dims, C.byref(n)))
    return tuple(int(d) for d in dims)


def fitting_dims(param: N4Param, shape):
    """Fitting-grid dimensions of a volume of ``shape`` (full size divided by
    the shrink factor), after the same size checks ``N4`` makes; raises
    ``N4Error`` for a volume ``N4`` would reject.  Needs no GPU."""
    dims = (C.c_uint * 3)()
    c = param.to_c()
    fx, fy, fz = (int(d) for d in shape)
    check(_lib.load().n4_fitting_dims(C.byref(c), fx, fy, fz, dims))
    return tuple(int(d) for d in dims)


# ---------------------------------------------------------------- context
class Context:
    """Owns the device workspaces of n4b200 (``n4_create`` / ``n4_destroy``)."""

    _default = {}

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        self.device = device
        check(_lib.load().n4_create(C.byref(self._h), device))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib.load().n4_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_profiling(self, enable: bool = True):
        check(_lib.load().n4_set_profiling(self._h, int(bool(enable))))

    def last_timings(self) -> dict:
        t = _lib.n4_timings_t()
        check(_lib.load().n4_last_timings(self._h, C.byref(t)))
        return dict(stage_ms=list(t.stage_ms), launches=t.launches, fit_voxels=t.fit_voxels,
                    full_voxels=t.full_voxels, fit_rows=t.fit_rows, fit_step=t.fit_step,
                    fit_depth=t.fit_depth,
                    correct_rows=t.correct_rows, correct_threads=t.correct_threads)

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = cls(device)
        return cls._default[device]


def _torch():
    import torch
    return torch


def _is_cuda(x) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


def _dev_f32(x, device=None):
    """CUDA float32 contiguous tensor view/copy of x (numpy or tensor)."""
    torch = _torch()
    if isinstance(x, torch.Tensor):
        t = x
        if not t.is_cuda:
            t = t.to(device or "cuda")
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.float32))).to(device or "cuda")
    if t.dtype != torch.float32:
        t = t.float()
    return t.contiguous()


def _dev_mask(m, device=None):
    """CUDA mask tensor and whether it is a byte mask: bool/uint8 input stays
    one byte per voxel (``N4_FLAG_MASK_U8``), anything else becomes float32."""
    torch = _torch()
    if m is None:
        return None, None
    if isinstance(m, torch.Tensor):
        t = m if m.is_cuda else m.to(device or "cuda")
        if t.dtype in (torch.uint8, torch.bool):
            return t.to(torch.uint8).contiguous(), True
        return (t if t.dtype == torch.float32 else t.float()).contiguous(), False
    a = np.asarray(m)
    if a.dtype in (np.uint8, np.bool_):
        return torch.from_numpy(np.ascontiguousarray(a.astype(np.uint8))).to(device or "cuda"), True
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(device or "cuda"), False


def _mask_flag(kinds) -> int:
    """N4_FLAG_MASK_U8 when the (non-None) masks of a call are byte masks."""
    k = {x for x in kinds if x is not None}
    if len(k) > 1:
        raise ValueError("the masks of one call must all be byte masks or all float masks")
    return _lib.FLAG_MASK_U8 if k == {True} else 0


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(device=None) -> int:
    return _torch().cuda.current_stream(device).cuda_stream


def _ctx_for(t, ctx):
    return ctx or Context.default(t.device.index or 0)


# ---------------------------------------------------------------- N4
@dataclass
class N4Result:
    im_normalized: object
    lattice: object
    bias_field: object = None
    report: dict = field(default_factory=dict)


def _report_dict(r: n4_report_t) -> dict:
    lv = r.levels
    return dict(status=_lib.STATUS.get(r.status, r.status), levels=lv,
                iterations=list(r.iterations[:lv]), final_cv=list(r.final_cv[:lv]),
                warm_start_used=bool(r.warm_start_used), first_cv_warm=r.first_cv_warm,
                first_cv_plain=r.first_cv_plain, foreground=r.foreground,
                path={1: "cluster", 2: "grid"}.get(r.path, r.path), cluster_size=r.cluster_size,
                device_begin_ns=int(r.device_begin_ns), device_end_ns=int(r.device_end_ns), sm=int(r.sm))


def N4(im, mask=None, param: Optional[N4Param] = None, warm_lattice=None, return_bias=False,
       ctx: Optional[Context] = None, synchronous: bool = True) -> N4Result:
    """Bias-correct one volume.

    ``im``/``mask``: float32 ``[fx][fy][fz]`` (mask != 0 is foreground; a
    bool/uint8 mask is passed as bytes; None = every voxel).  CUDA tensors run on their device and stream; numpy arrays
    take the host path (``n4_run_host``).  Returns the corrected volume, the
    final control lattice and, with ``return_bias``, ``exp(log bias)``.
    """
    param = param or N4Param()
    cpar = param.to_c()
    fx, fy, fz = (int(d) for d in im.shape)
    dims = lattice_dims(param)
    lib = _lib.load()
    rep = n4_report_t()
    if _is_cuda(im):
        torch = _torch()
        imt = _dev_f32(im)
        mk, u8 = _dev_mask(mask, imt.device)
        cpar.flags |= _mask_flag([u8])
        wl = None if warm_lattice is None else _dev_f32(warm_lattice, imt.device)
        out = torch.empty_like(imt)
        lat = torch.empty(dims, dtype=torch.float32, device=imt.device)
        bias = torch.empty_like(imt) if return_bias else None
        c = _ctx_for(imt, ctx)
        st = lib.n4_run(c.handle, C.byref(cpar), _ptr(imt), _ptr(mk), fx, fy, fz, _ptr(out), _ptr(lat),
                        _ptr(bias), _ptr(wl), _stream(imt.device), C.byref(rep) if synchronous else None)
        check(st)
        return N4Result(out, lat, bias, _report_dict(rep) if synchronous else {})
    imh = np.ascontiguousarray(np.asarray(im, dtype=np.float32))
    mkh = None
    if mask is not None:
        ma = np.asarray(mask)
        if ma.dtype in (np.uint8, np.bool_):
            mkh = np.ascontiguousarray(ma.astype(np.uint8))
            cpar.flags |= _lib.FLAG_MASK_U8
        else:
            mkh = np.ascontiguousarray(ma, dtype=np.float32)
    wlh = None if warm_lattice is None else np.ascontiguousarray(np.asarray(warm_lattice, dtype=np.float32))
    out = np.empty_like(imh)
    lat = np.empty(dims, dtype=np.float32)
    bias = np.empty_like(imh) if return_bias else None
    c = ctx or Context.default(0)
    p = lambda a: None if a is None else a.ctypes.data
    st = lib.n4_run_host(c.handle, C.byref(cpar), p(imh), p(mkh), fx, fy, fz, p(out), p(lat), p(bias), p(wlh),
                         C.byref(rep))
    check(st)
    return N4Result(out, lat, bias, _report_dict(rep))


def N4Batch(volumes: Sequence, param: Optional[N4Param] = None, warm_lattices=None, return_bias=False,
            ctx: Optional[Context] = None, synchronous: bool = True, encoder=None):
    """Bias-correct many volumes (CUDA tensors, any sizes) in one persistent
    launch.  ``volumes``: sequence of ``(im, mask)``.  With ``encoder`` (an
    ``n4b200.encoder.Encoder``) the first-level lattices are predicted inside
    the run (``n4_run_batched_warm``).  Returns a list of ``N4Result``."""
    torch = _torch()
    param = param or N4Param()
    cpar = param.to_c()
    kinds = []
    dims = lattice_dims(param)
    n = len(volumes)
    arr = (n4_volume_t * n)()
    keep, results = [], []
    dev = None
    for i, (im, mask) in enumerate(volumes):
        imt = _dev_f32(im)
        dev = imt.device
        mk, u8 = _dev_mask(mask, dev)
        kinds.append(u8)
        wl = None if warm_lattices is None or warm_lattices[i] is None else _dev_f32(warm_lattices[i], dev)
        out = torch.empty_like(imt)
        lat = torch.empty(dims, dtype=torch.float32, device=dev)
        bias = torch.empty_like(imt) if return_bias else None
        keep += [imt, mk, wl]
        fx, fy, fz = (int(d) for d in imt.shape)
        arr[i] = n4_volume_t(_ptr(imt), _ptr(mk), fx, fy, fz, _ptr(out), _ptr(lat), _ptr(bias), _ptr(wl))
        results.append(N4Result(out, lat, bias, {}))
    cpar.flags |= _mask_flag(kinds)
    reps = (n4_report_t * n)()
    c = ctx or Context.default(dev.index or 0)
    if encoder is not None:
        st = _lib.load().n4_run_batched_warm(c.handle, C.byref(cpar), n, arr, encoder.h, _stream(dev),
                                             reps if synchronous else None)
    else:
        st = _lib.load().n4_run_batched(c.handle, C.byref(cpar), n, arr, _stream(dev), reps if synchronous else None)
    check(st)
    if synchronous:
        for r, rep in zip(results, reps):
            r.report = _report_dict(rep)
    return results


def N4BatchHost(volumes: Sequence, param: Optional[N4Param] = None, per: int = 0, encoder=None,
                return_bias: bool = False, outputs=None, ctx: Optional[Context] = None, device: int = 0):
    """Bias-correct volumes held in host memory (``n4_run_batched_host``):
    uploads, batched runs and downloads overlap over sub-batches of ``per``
    volumes.  ``volumes``: sequence of ``(im, mask)`` CPU tensors (page-locked
    for overlapped copies; float32 images, float32 or uint8 masks, or None).
    ``outputs``: optional preallocated ``(im_normalized, lattice)`` CPU
    tensors per volume.  Returns ``(results, device_ms)``: a list of
    ``N4Result`` with host tensors, and the GPU time from the first upload to
    the last download."""
    torch = _torch()
    param = param or N4Param()
    cpar = param.to_c()
    dims = lattice_dims(param)
    n = len(volumes)
    arr = (n4_volume_t * n)()
    keep, results, kinds = [], [], []
    for i, (im, mask) in enumerate(volumes):
        imt = torch.as_tensor(im)
        if imt.is_cuda or imt.dtype != torch.float32 or not imt.is_contiguous():
            raise ValueError("N4BatchHost takes contiguous float32 CPU images")
        mk = None
        if mask is not None:
            mk = torch.as_tensor(mask)
            if mk.is_cuda or mk.dtype not in (torch.float32, torch.uint8) or not mk.is_contiguous():
                raise ValueError("masks must be contiguous float32 or uint8 CPU tensors")
            kinds.append(mk.dtype == torch.uint8)
        if outputs is not None:
            out, lat = outputs[i]
        else:
            out = torch.empty(imt.shape, dtype=torch.float32, pin_memory=True)
            lat = torch.empty(dims, dtype=torch.float32, pin_memory=True)
        bias = torch.empty(imt.shape, dtype=torch.float32, pin_memory=True) if return_bias else None
        keep += [imt, mk, out, lat, bias]
        fx, fy, fz = (int(d) for d in imt.shape)
        arr[i] = n4_volume_t(imt.data_ptr(), None if mk is None else mk.data_ptr(), fx, fy, fz, out.data_ptr(),
                             lat.data_ptr(), None if bias is None else bias.data_ptr(), None)
        results.append(N4Result(out, lat, bias, {}))
    if kinds and len(set(kinds)) > 1:
        raise ValueError("all masks of a batch must have one type")
    if kinds and kinds[0]:
        cpar.flags |= _lib.FLAG_MASK_U8
    reps = (n4_report_t * n)()
    ms = C.c_float()
    c = ctx or Context.default(device)
    check(_lib.load().n4_run_batched_host(c.handle, C.byref(cpar), n, arr, int(per),
                                          None if encoder is None else encoder.h, reps, C.byref(ms)))
    for r, rep in zip(results, reps):
        r.report = _report_dict(rep)
    return results, float(ms.value)


def warm_inputs(volumes: Sequence, param: Optional[N4Param] = None, ctx: Optional[Context] = None):
    """Network inputs of the learned warm start (``n4_warm_inputs``): every
    volume's masked log fitting grid pooled to 32x32x24, CUDA BF16
    ``[n, 32, 32, 24]``."""
    torch = _torch()
    param = param or N4Param()
    cpar = param.to_c()
    kinds = []
    n = len(volumes)
    arr = (n4_volume_t * n)()
    keep = []
    dev = None
    for i, (im, mask) in enumerate(volumes):
        imt = _dev_f32(im)
        dev = imt.device
        mk, u8 = _dev_mask(mask, dev)
        kinds.append(u8)
        keep += [imt, mk]
        fx, fy, fz = (int(d) for d in imt.shape)
        arr[i] = n4_volume_t(_ptr(imt), _ptr(mk), fx, fy, fz, None, None, None, None)
    cpar.flags |= _mask_flag(kinds)
    x = torch.empty((n, 32, 32, 24), dtype=torch.bfloat16, device=dev)
    c = ctx or Context.default(dev.index or 0)
    check(_lib.load().n4_warm_inputs(c.handle, C.byref(cpar), n, arr, x.data_ptr(), _stream(dev)))
    return x


def cluster_size_flag(k: int) -> int:
    """``N4_FLAG_CLUSTER_SIZE(k)``: run the cluster path with k CTAs per volume."""
    return (int(k) & 31) << 8


def autotune(volumes: Sequence, param: Optional[N4Param] = None, ctx: Optional[Context] = None) -> dict:
    """Time every execution configuration that fits these volumes
    (``n4_autotune``) and record the fastest in the context for later runs
    of volumes of the same sizes with the same lattice, levels and bins.
    Returns ``{"candidates": [(cluster_size, threads, ms), ...], "chosen":
    cluster_size, "chosen_threads": threads, "correction": [(rows, threads,
    ms), ...], "correction_chosen": (rows, threads), "sub_batches_ms":
    [(count, tapered, adapt, ms), ...], "sub_batches_chosen": (count,
    tapered, adapt)}`` (cluster size 0 = whole-GPU path; the correction tile
    shapes and the sub-batch splits are timed on the chosen path; adapt > 0:
    each sub-batch on the smallest cluster size >= adapt that holds its
    volumes, 0: every sub-batch on the chosen size)."""
    torch = _torch()
    param = param or N4Param()
    cpar = param.to_c()
    kinds = []
    dims = lattice_dims(param)
    n = len(volumes)
    arr = (n4_volume_t * n)()
    keep = []
    dev = None
    for i, (im, mask) in enumerate(volumes):
        imt = _dev_f32(im)
        dev = imt.device
        mk, u8 = _dev_mask(mask, dev)
        kinds.append(u8)
        out = torch.empty_like(imt)
        lat = torch.empty(dims, dtype=torch.float32, device=dev)
        keep += [imt, mk, out, lat]
        fx, fy, fz = (int(d) for d in imt.shape)
        arr[i] = n4_volume_t(_ptr(imt), _ptr(mk), fx, fy, fz, _ptr(out), _ptr(lat), None, None)
    cpar.flags |= _mask_flag(kinds)
    c = ctx or Context.default(dev.index or 0)
    rep = _lib.n4_tune_report_t()
    check(_lib.load().n4_autotune(c.handle, C.byref(cpar), n, arr, _stream(dev), C.byref(rep)))
    cands = [(int(rep.cluster_size[k]), int(rep.threads[k]), float(rep.ms[k])) for k in range(rep.candidates)]
    corr = [(int(rep.corr_rows[k]), int(rep.corr_threads[k]), float(rep.corr_ms[k]))
            for k in range(rep.corr_candidates)]
    subs = [(int(rep.sub_count[k]), bool(rep.sub_tapered[k]), int(rep.sub_adapt[k]), float(rep.sub_ms[k]))
            for k in range(rep.sub_candidates)]
    return {"candidates": cands, "chosen": cands[rep.chosen][0], "chosen_threads": cands[rep.chosen][1],
            "correction": corr, "correction_chosen": corr[rep.corr_chosen][:2] if corr else None,
            "sub_batches_ms": subs, "sub_batches_chosen": subs[rep.sub_chosen][:3] if subs else None}


def autotune_components(field, mask, numberOfControlPoints, ctx: Optional[Context] = None) -> dict:
    """Time the tile shapes of the standalone fit (``FitBspline3D``) and of
    the dense evaluation (``EvaluateBspline3D``) on this field and lattice
    size (``n4_autotune_components``) and record the fastest of each in the
    context; later calls with the same sizes use them.  Returns the timed
    candidates and the chosen shapes."""
    torch = _torch()
    f = _dev_f32(field)
    m = None if mask is None else _dev_f32(mask, f.device)
    nc = tuple(int(c) for c in numberOfControlPoints)
    lat = torch.empty(nc, dtype=torch.float32, device=f.device)
    out = torch.empty_like(f)
    c = ctx or Context.default(f.device.index or 0)
    rep = _lib.n4_component_tune_t()
    X, Y, Z = (int(d) for d in f.shape)
    check(_lib.load().n4_autotune_components(c.handle, _ptr(f), _ptr(m), *nc, X, Y, Z, _ptr(lat), _ptr(out),
                                             _stream(f.device), C.byref(rep)))
    fit = [(int(rep.fit_step[k]), int(rep.fit_depth[k]), int(rep.fit_rows[k]), float(rep.fit_ms[k]))
           for k in range(rep.fit_candidates)]
    ev = [(int(rep.eval_rows[k]), int(rep.eval_threads[k]), float(rep.eval_ms[k])) for k in range(rep.eval_candidates)]
    return {"fit": fit, "fit_chosen": fit[rep.fit_chosen][:3], "evaluate": ev,
            "evaluate_chosen": ev[rep.eval_chosen][:2]}


class N4BatchGraph:
    """A batched run recorded once as a CUDA graph and replayed with
    ``launch()`` (``n4_batch_graph_*``).  Inputs are read from the given
    CUDA tensors at every launch (refill them in place to correct new data);
    outputs are written to ``results[i].im_normalized`` etc.
    ``kernel_launches``: the library's kernels per launch; ``sub_batches``:
    how many sub-batches the run overlaps (``N4_FLAG_SUB_BATCHES``)."""

    def __init__(self, volumes: Sequence, param: Optional[N4Param] = None, warm_lattices=None,
                 return_bias=False, ctx: Optional[Context] = None, encoder=None):
        torch = _torch()
        param = param or N4Param()
        self._cpar = param.to_c()
        kinds = []
        dims = lattice_dims(param)
        n = len(volumes)
        arr = (n4_volume_t * n)()
        self._keep, self.results = [], []
        dev = None
        for i, (im, mask) in enumerate(volumes):
            imt = _dev_f32(im)
            dev = imt.device
            mk, u8 = _dev_mask(mask, dev)
            kinds.append(u8)
            wl = None if warm_lattices is None or warm_lattices[i] is None else _dev_f32(warm_lattices[i], dev)
            out = torch.empty_like(imt)
            lat = torch.empty(dims, dtype=torch.float32, device=dev)
            bias = torch.empty_like(imt) if return_bias else None
            self._keep += [imt, mk, wl]
            fx, fy, fz = (int(d) for d in imt.shape)
            arr[i] = n4_volume_t(_ptr(imt), _ptr(mk), fx, fy, fz, _ptr(out), _ptr(lat), _ptr(bias), _ptr(wl))
            self.results.append(N4Result(out, lat, bias, {}))
        self._cpar.flags |= _mask_flag(kinds)
        self.inputs = [(self._keep[3 * i], self._keep[3 * i + 1]) for i in range(n)]
        self.ctx = ctx or Context.default(dev.index or 0)
        self.device = dev
        self._h = C.c_void_p()
        self.encoder = encoder
        if encoder is not None:
            check(_lib.load().n4_batch_graph_create_warm(self.ctx.handle, C.byref(self._cpar), n, arr, encoder.h,
                                                         C.byref(self._h)))
        else:
            check(_lib.load().n4_batch_graph_create(self.ctx.handle, C.byref(self._cpar), n, arr,
                                                    C.byref(self._h)))
        nl, ns = C.c_int(), C.c_int()
        check(_lib.load().n4_batch_graph_info(self._h, C.byref(nl), C.byref(ns)))
        self.kernel_launches, self.sub_batches = nl.value, ns.value

    def launch(self):
        check(_lib.load().n4_batch_graph_launch(self._h, _stream(self.device)))

    def sync(self):
        n = len(self.results)
        reps = (n4_report_t * n)()
        check(_lib.load().n4_batch_graph_sync(self._h, reps, n))
        for r, rep in zip(self.results, reps):
            r.report = _report_dict(rep)
        return self.results

    def close(self):
        if self._h:
            _lib.load().n4_batch_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- components
def _out_like(x, t):
    return t if _is_cuda(x) else t.cpu().numpy()


def FitBspline3D(field, mask, numberOfControlPoints, eps: float = 1e-3, zero_den: bool = False,
                 ctx: Optional[Context] = None):
    """Lattice fitted to ``field`` over ``mask != 0`` (``N4.py:186-237``;
    ``zero_den`` gives ``cudaN4.cu:123-127``'s division)."""
    torch = _torch()
    f = _dev_f32(field)
    m = None if mask is None else _dev_f32(mask, f.device)
    nc = tuple(int(c) for c in numberOfControlPoints)
    lat = torch.empty(nc, dtype=torch.float32, device=f.device)
    X, Y, Z = f.shape
    check(_lib.load().n4_fit_bspline3d(_ctx_for(f, ctx).handle, _ptr(f), _ptr(m), *nc, X, Y, Z, float(eps),
                                       int(bool(zero_den)), _ptr(lat), _stream(f.device)))
    return _out_like(field, lat)


def EvaluateBspline3D(lattice, numberOfControlPoints, size, ctx: Optional[Context] = None):
    """Dense evaluation of the lattice on ``size`` voxels (``N4.py:241-273``)."""
    torch = _torch()
    L = _dev_f32(lattice)
    nc = tuple(int(c) for c in numberOfControlPoints)
    X, Y, Z = (int(s) for s in size)
    out = torch.empty((X, Y, Z), dtype=torch.float32, device=L.device)
    check(_lib.load().n4_evaluate_bspline3d(_ctx_for(L, ctx).handle, _ptr(L), *nc, X, Y, Z, _ptr(out),
                                            _stream(L.device)))
    return _out_like(lattice, out)


def UpsampleLattice3D(lattice, ctx: Optional[Context] = None):
    """(n+3) -> (2n+3) control points per axis (``N4.py:132-165``)."""
    torch = _torch()
    L = _dev_f32(lattice)
    nx, ny, nz = (int(s) for s in L.shape)
    out = torch.empty((2 * nx - 3, 2 * ny - 3, 2 * nz - 3), dtype=torch.float32, device=L.device)
    check(_lib.load().n4_upsample_lattice3d(_ctx_for(L, ctx).handle, _ptr(L), nx, ny, nz, _ptr(out),
                                            _stream(L.device)))
    return _out_like(lattice, out)


upsampleLattice3D = UpsampleLattice3D


def sharpenImage(im_before_sharpen, mask, numberOfHistogramBins: int = 200, WienerFilterNoise: float = 0.01,
                 BiasFieldFullWidthAtHalfMaximum: float = 0.15, details: bool = False,
                 ctx: Optional[Context] = None):
    """Histogram sharpening of a log image over the mask (``N4.py:9-118``).
    With ``details`` also returns ``dict(binMin, binMax, E)``."""
    torch = _torch()
    x = _dev_f32(im_before_sharpen)
    m = None if mask is None else _dev_f32(mask, x.device)
    out = torch.empty_like(x)
    bmin, bmax = C.c_float(), C.c_float()
    E = np.zeros(int(numberOfHistogramBins), dtype=np.float32)
    torch.cuda.synchronize(x.device)
    check(_lib.load().n4_sharpen_image(_ctx_for(x, ctx).handle, _ptr(x), _ptr(m), x.numel(),
                                       int(numberOfHistogramBins), float(WienerFilterNoise),
                                       float(BiasFieldFullWidthAtHalfMaximum), _ptr(out), C.byref(bmin),
                                       C.byref(bmax), E.ctypes.data))
    res = _out_like(im_before_sharpen, out)
    if details:
        return res, dict(binMin=bmin.value, binMax=bmax.value, E=E)
    return res


def CalculateConvergenceMeasurement(field1, field2, mask, ddof: int = 0, ctx: Optional[Context] = None) -> float:
    """std / mean of exp(field1 - field2) over the mask (``N4.py:121-126``;
    ``ddof=1`` is ``cudaN4.cu:979``)."""
    a = _dev_f32(field1)
    b = _dev_f32(field2, a.device)
    m = None if mask is None else _dev_f32(mask, a.device)
    out = C.c_double()
    _torch().cuda.synchronize(a.device)
    check(_lib.load().n4_convergence(_ctx_for(a, ctx).handle, _ptr(a), _ptr(b), _ptr(m), a.numel(), int(ddof),
                                     C.byref(out)))
    return out.value


calculateConvergenceMeasurement = CalculateConvergenceMeasurement
