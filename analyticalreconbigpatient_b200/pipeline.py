"""Whole-scan reconstruction through the library's chain plan.

``HelicalRecon`` wraps ``hr_recon_plan`` (csrc/recon.cpp), which restates the
per-segment driver src/analyticalReconBigPatient.m:77-146 for a whole scan
held in HBM: rebin, drop the half-fan margin at the scan ends (m-file
:80-93), preweight + ramp filter, backproject. The plan's geometry tables and
intermediate buffers are made once; ``run`` only enqueues kernels on a stream
(timed or captured by the caller), ``run_host`` copies host data in and the
volume out around it.

``StagePlans`` exposes the three stage plans separately (used for the FP64
data path and for per-stage timing).

PyTorch provides device memory and streams only; all compute runs in
libhelixrecon.so.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .geometry import Scan


def _stream(device: torch.device, stream) -> int:
    if stream is None:
        return torch.cuda.current_stream(device).cuda_stream
    return stream if isinstance(stream, int) else stream.cuda_stream


def recon_desc(scan: Scan, w: np.ndarray, form: int) -> _lib.ReconDesc:
    ra, fa = scan.rebin_args(), scan.filter_args()
    return _lib.ReconDesc(YL=ra["YL"], ZL=ra["ZL"], ViewN=ra["ViewN"], YLC=ra["YLC"], dYA=ra["dYA"],
                          DeltaTheta=ra["DeltaTheta"], PLC=ra["PLC"], DeltaT=ra["DeltaT"], DeltaFai=ra["DeltaFai"],
                          SO=ra["SO"], view0=scan.crop_front, fPLC=fa["PLC"], fZLC=fa["ZLC"], fdYL=fa["dYL"],
                          fdZL=fa["dZL"], fSO=fa["SO"], bp=_lib.BpGeom.from_dict(scan.bp_geom()), w=w.ctypes.data,
                          form=form)


def view_weights(scan: Scan) -> np.ndarray:
    w = np.zeros(scan.N_2pi, dtype=np.float64)
    _lib.call("hr_view_weights", w.ctypes.data, scan.N_2pi, scan.HSCoef, scan.delta)
    return w


class HelicalRecon:
    """Whole-scan reconstruction on one GPU (float volume)."""

    def __init__(self, scan: Scan, form: int = _lib.HR_FORM_PLAIN, device: int | torch.device = 0):
        self.scan = scan
        self.form = form
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self._plan = ctypes.c_void_p()
        w = view_weights(scan)
        desc = recon_desc(scan, w, form)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_recon_plan_create(ctypes.byref(self._plan), ctypes.byref(desc)))
        self.volume = torch.empty((scan.YN, scan.XN, scan.ZN), dtype=torch.float32, device=self.device)

    @property
    def device_bytes(self) -> int:
        return int(_lib.load().hr_recon_device_bytes(self._plan))

    def check(self) -> None:
        """Raise if a kernel of an earlier execution reported a timed-out pipeline wait (synchronises)."""
        _lib.check(_lib.load().hr_recon_check(self._plan))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        _lib.check(_lib.load().hr_recon_describe(self._plan, buf, 1024))
        return buf.value.decode()

    def run(self, fan: torch.Tensor, volume: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """fan: device float32 [views][YL][ZL] (post-flip channel order)."""
        vol = self.volume if volume is None else volume
        if fan.dtype != torch.float32 or not fan.is_contiguous() or fan.numel() != self.scan.projection_bytes() // 4:
            raise ValueError("fan must be a contiguous float32 tensor of [views][YL][ZL]")
        _lib.check(_lib.load().hr_recon_execute(self._plan, vol.data_ptr(), fan.data_ptr(), _stream(self.device,
                                                                                                      stream)))
        return vol

    def run_host(self, fan, volume=None):
        """Host arrays (numpy or CPU tensors; pinned for full copy speed); either may also be a CUDA
        tensor (a host fan into a device volume, for instance). Synchronous."""
        s = self.scan
        if volume is None:
            volume = np.empty((s.YN, s.XN, s.ZN), dtype=np.float32)
        fp = fan.data_ptr() if isinstance(fan, torch.Tensor) else np.ascontiguousarray(fan, np.float32).ctypes.data
        vp = volume.data_ptr() if isinstance(volume, torch.Tensor) else volume.ctypes.data
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_recon_execute_host(self._plan, vp, fp))
        return volume

    def close(self) -> None:
        if self._plan:
            _lib.load().hr_recon_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def slab_windows(scan: Scan, slab_slices: int, part: int = 0, nparts: int = 1,
                 assign: int = _lib.HR_SLAB_BLOCKS) -> list[dict]:
    """Slab windows of part ``part`` of ``nparts`` (hr_slab_windows: host
    arithmetic only, no GPU needed): one dict per slab with its slices, its
    backprojection window (cropped, rebinned view numbering) and its fan window."""
    w = view_weights(scan)
    desc = recon_desc(scan, w, _lib.HR_FORM_FAST)
    lib = _lib.load()
    n = ctypes.c_int(0)
    _lib.check(lib.hr_slab_windows(ctypes.byref(desc), slab_slices, part, nparts, assign, None, 0, ctypes.byref(n)))
    arr = (_lib.SlabWindow * max(1, n.value))()
    _lib.check(lib.hr_slab_windows(ctypes.byref(desc), slab_slices, part, nparts, assign, arr, n.value,
                                   ctypes.byref(n)))
    return [{k: getattr(arr[i], k) for k, _ in _lib.SlabWindow._fields_} for i in range(n.value)]


def plain_slab(scan: Scan, win: dict, fan_window: torch.Tensor) -> torch.Tensor:
    """The plain FP32 chain (the drop-in numerics) on one slab of a long scan:
    the slab's fan window ``fan_window`` [fan_views][YL][ZL] (on the device) is
    rebinned with the whole scan's rebinning arguments, its backprojection
    window filtered and backprojected into the slab's slices. Returns the slab
    [YN][XN][n_slices]. The reference the slab pipeline's per-slab error is
    stated against."""
    lib = _lib.load()
    ra, fa = scan.rebin_args(), scan.filter_args()
    g = scan.bp_geom()
    gs = dict(g, ZN=win["n_slices"], ZNC=g["ZNC"] - win["first_slice"], PN=win["bp_views"],
              BetaS=g["BetaS"] + win["bp_view0"] * g["DeltaFai"])
    dev = fan_window.device
    reb, filt, bp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    w = view_weights(scan)
    geom = _lib.BpGeom.from_dict(gs)
    try:
        _lib.check(lib.hr_rebin_plan_create(ctypes.byref(reb), ra["YL"], ra["ZL"], win["fan_views"], ra["YLC"],
                                            ra["dYA"], ra["DeltaTheta"], ra["PLC"], ra["DeltaT"], ra["DeltaFai"],
                                            ra["SO"]))
        _lib.check(lib.hr_filter_plan_create(ctypes.byref(filt), fa["YL"], fa["ZL"], win["bp_views"], fa["PLC"],
                                             fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"]))
        _lib.check(lib.hr_bp_plan_create(ctypes.byref(bp), ctypes.byref(geom), w.ctypes.data, _lib.HR_FORM_PLAIN))
        rebinned = torch.empty_like(fan_window)
        filtered = torch.empty((win["bp_views"], scan.ZL, scan.YL), dtype=torch.float32, device=dev)
        out = torch.empty((scan.YN, scan.XN, win["n_slices"]), dtype=torch.float32, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.hr_rebin_execute(reb, rebinned.data_ptr(), fan_window.data_ptr(), st))
        _lib.check(lib.hr_filter_execute(filt, filtered.data_ptr(), rebinned.data_ptr(), _lib.HR_LAYOUT_REBIN,
                                         scan.crop_front, st))
        _lib.check(lib.hr_bp_execute(bp, out.data_ptr(), filtered.data_ptr(), st))
        torch.cuda.synchronize(dev)
    finally:
        lib.hr_rebin_plan_destroy(reb)
        lib.hr_filter_plan_destroy(filt)
        lib.hr_bp_plan_destroy(bp)
    return out


class SlabRecon:
    """Long scans reconstructed slab by slab (disjoint z slabs, each from its own
    view window) through a captured CUDA graph; see hr_slab_plan in
    include/helixrecon.h. Fast form only. ``part``/``nparts`` split the slabs
    of one scan between GPUs (one plan per GPU, no exchange)."""

    def __init__(self, scan: Scan, slab_slices: int = 64, device: int | torch.device = 0, part: int = 0,
                 nparts: int = 1, assign: int = _lib.HR_SLAB_BLOCKS):
        self.scan = scan
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self._plan = ctypes.c_void_p()
        w = view_weights(scan)
        desc = recon_desc(scan, w, _lib.HR_FORM_FAST)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_slab_plan_create_part(ctypes.byref(self._plan), ctypes.byref(desc), slab_slices,
                                                            part, nparts, assign))

    def fan_range(self) -> tuple[int, int, int]:
        """(first fan view, view count, bytes copied from the fan per run)."""
        first, n, nbytes = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_size_t(0)
        _lib.check(_lib.load().hr_slab_fan_range(self._plan, ctypes.byref(first), ctypes.byref(n),
                                                 ctypes.byref(nbytes)))
        return first.value, n.value, nbytes.value

    def run(self, fan, volume, fan_view0: int = 0) -> None:
        """fan/volume: torch tensors (CUDA or CPU; pinned CPU tensors overlap copies with compute).
        ``fan`` holds fan views [fan_view0, ...) of the scan (at least the plan's fan_range)."""
        def ptr(t):
            return (t.data_ptr(), 0) if t.is_cuda else (t.data_ptr(), 1)
        fp, fh = ptr(fan)
        vp, vh = ptr(volume)
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_slab_execute_range(self._plan, vp, fp, fan_view0, vh, fh))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        _lib.check(_lib.load().hr_slab_describe(self._plan, buf, 1024))
        return buf.value.decode()

    @property
    def device_bytes(self) -> int:
        return int(_lib.load().hr_slab_device_bytes(self._plan))

    def close(self) -> None:
        if self._plan:
            _lib.load().hr_slab_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchRecon:
    """Several independent scans of uneven size; every scan's rebinning and
    tensor-core filter, then one persistent backprojection launch over all of
    them, replayed from a CUDA graph (hr_batch_plan in include/helixrecon.h).
    Fast form only; at most 16 scans."""

    def __init__(self, scans: list[Scan], device: int | torch.device = 0):
        self.scans = list(scans)
        self.device = torch.device("cuda", device) if isinstance(device, int) else device
        self._plan = ctypes.c_void_p()
        ws = [view_weights(sc) for sc in self.scans]  # alive until the plan has copied them
        descs = (_lib.ReconDesc * len(self.scans))(*[recon_desc(sc, w, _lib.HR_FORM_FAST)
                                                    for sc, w in zip(self.scans, ws)])
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_batch_plan_create(ctypes.byref(self._plan), descs, len(self.scans)))

    def run(self, fans: list[torch.Tensor], volumes: list[torch.Tensor], stream=None) -> None:
        """fans[i]: CUDA float32 [views][YL][ZL]; volumes[i]: CUDA float32 [YN][XN][ZN]."""
        n = len(self.scans)
        if len(fans) != n or len(volumes) != n:
            raise ValueError(f"expected {n} fans and volumes")
        for sc, f, v in zip(self.scans, fans, volumes):
            if not (f.is_cuda and v.is_cuda and f.dtype == torch.float32 and v.dtype == torch.float32):
                raise TypeError("fans and volumes must be CUDA float32 tensors")
            if tuple(f.shape) != (sc.views, sc.YL, sc.ZL) or tuple(v.shape) != (sc.YN, sc.XN, sc.ZN):
                raise ValueError("fan or volume shape does not match its scan")
        fp = (ctypes.c_void_p * n)(*[f.data_ptr() for f in fans])
        vp = (ctypes.c_void_p * n)(*[v.data_ptr() for v in volumes])
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_batch_execute(self._plan, vp, fp, _stream(self.device, stream)))

    def run_host(self, fans: list[torch.Tensor], volumes: list[torch.Tensor]) -> None:
        """The batch from host memory, synchronous (hr_batch_execute_host): fans[i]
        CPU float32 [views][YL][ZL] (page-locked for copies that overlap the
        computation), volumes[i] CPU float32 [YN][XN][ZN], written in place."""
        n = len(self.scans)
        if len(fans) != n or len(volumes) != n:
            raise ValueError(f"expected {n} fans and volumes")
        for sc, f, v in zip(self.scans, fans, volumes):
            if f.is_cuda or v.is_cuda or f.dtype != torch.float32 or v.dtype != torch.float32:
                raise TypeError("fans and volumes must be CPU float32 tensors")
            if not (f.is_contiguous() and v.is_contiguous()):
                raise ValueError("fans and volumes must be contiguous")
            if tuple(f.shape) != (sc.views, sc.YL, sc.ZL) or tuple(v.shape) != (sc.YN, sc.XN, sc.ZN):
                raise ValueError("fan or volume shape does not match its scan")
        fp = (ctypes.c_void_p * n)(*[f.data_ptr() for f in fans])
        vp = (ctypes.c_void_p * n)(*[v.data_ptr() for v in volumes])
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_batch_execute_host(self._plan, vp, fp))

    def backproject(self, volumes: list[torch.Tensor], stream=None) -> None:
        """Only the persistent backprojection, from the filtered data of the last run."""
        vp = (ctypes.c_void_p * len(self.scans))(*[v.data_ptr() for v in volumes])
        with torch.cuda.device(self.device):
            _lib.check(_lib.load().hr_batch_backproject(self._plan, vp, _stream(self.device, stream)))

    def select(self, variant: int) -> None:
        _lib.check(_lib.load().hr_batch_select(self._plan, variant))

    def check(self) -> None:
        _lib.check(_lib.load().hr_batch_check(self._plan))

    def describe(self) -> str:
        buf = ctypes.create_string_buffer(1024)
        _lib.check(_lib.load().hr_batch_describe(self._plan, buf, 1024))
        return buf.value.decode()

    @property
    def device_bytes(self) -> int:
        return int(_lib.load().hr_batch_device_bytes(self._plan))

    def close(self) -> None:
        if self._plan:
            _lib.load().hr_batch_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class StagePlans:
    """The three stage plans of a scan, for per-stage use and the FP64 form."""

    def __init__(self, scan: Scan, form: int = _lib.HR_FORM_PLAIN):
        lib = _lib.load()
        self.scan, self.form = scan, form
        self._rebin, self._filter, self._bp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        ra, fa = scan.rebin_args(), scan.filter_args()
        _lib.check(lib.hr_rebin_plan_create(ctypes.byref(self._rebin), ra["YL"], ra["ZL"], ra["ViewN"], ra["YLC"],
                                            ra["dYA"], ra["DeltaTheta"], ra["PLC"], ra["DeltaT"], ra["DeltaFai"],
                                            ra["SO"]))
        _lib.check(lib.hr_filter_plan_create(ctypes.byref(self._filter), fa["YL"], fa["ZL"], fa["ViewN"], fa["PLC"],
                                             fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"]))
        self.w = view_weights(scan)
        geom = _lib.BpGeom.from_dict(scan.bp_geom())
        _lib.check(lib.hr_bp_plan_create(ctypes.byref(self._bp), ctypes.byref(geom), self.w.ctypes.data, form))
        self._filter_tc = ctypes.c_void_p()
        if form == _lib.HR_FORM_FAST:
            _lib.check(lib.hr_filter_tc_plan_create(ctypes.byref(self._filter_tc), fa["YL"], fa["ZL"], fa["ViewN"],
                                                    fa["PLC"], fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"]))

    def rebin(self, out: torch.Tensor, fan: torch.Tensor, stream: int = 0) -> None:
        _lib.check(_lib.load().hr_rebin_execute(self._rebin, out.data_ptr(), fan.data_ptr(), stream))

    def filter(self, out: torch.Tensor, inp: torch.Tensor, in_layout: int, view0: int, stream: int = 0) -> None:
        _lib.check(_lib.load().hr_filter_execute(self._filter, out.data_ptr(), inp.data_ptr(), in_layout, view0,
                                                 stream))

    def backproject(self, vol: torch.Tensor, fp: torch.Tensor, stream: int = 0) -> None:
        _lib.check(_lib.load().hr_bp_execute(self._bp, vol.data_ptr(), fp.data_ptr(), stream))

    def filter_tc(self, pairs: torch.Tensor, inp: torch.Tensor, in_layout: int, view0: int, stream: int = 0) -> None:
        """Tensor-core Toeplitz filter straight to BF16 channel pairs (fast form)."""
        _lib.check(_lib.load().hr_filter_tc_execute(self._filter_tc, pairs.data_ptr(), inp.data_ptr(), in_layout,
                                                    view0, stream))

    def check(self) -> None:
        if self._filter_tc:
            _lib.check(_lib.load().hr_filter_tc_check(self._filter_tc))

    def autotune(self, vol: torch.Tensor, fp: torch.Tensor, stream: int = 0) -> str:
        lib = _lib.load()
        _lib.check(lib.hr_bp_autotune(self._bp, vol.data_ptr(), fp.data_ptr(), stream))
        buf = ctypes.create_string_buffer(1024)
        _lib.check(lib.hr_bp_describe(self._bp, buf, 1024))
        return buf.value.decode()

    def pack(self, out: torch.Tensor, filtered: torch.Tensor, stream: int = 0) -> None:
        """FP32 filtered rows -> BF16 channel pairs (the fast form's layout)."""
        s = self.scan
        _lib.check(_lib.load().hr_pack_bf16_pairs(out.data_ptr(), filtered.data_ptr(), s.ZL * s.PN, s.YL, stream))

    def close(self) -> None:
        lib = _lib.load()
        for attr, fn in (("_rebin", lib.hr_rebin_plan_destroy), ("_filter", lib.hr_filter_plan_destroy),
                         ("_bp", lib.hr_bp_plan_destroy), ("_filter_tc", lib.hr_filter_tc_plan_destroy)):
            if getattr(self, attr, None):
                fn(getattr(self, attr))
                setattr(self, attr, ctypes.c_void_p())

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def project(scan: Scan, objects: np.ndarray, out: torch.Tensor | None = None, device: int = 0) -> torch.Tensor:
    """Analytic fan projections of a phantom on the GPU: float32 [views][YL][ZL]."""
    from .phantom import projector_args

    dev = torch.device("cuda", device)
    a = projector_args(scan)
    if out is None:
        out = torch.empty((a["ViewN"], a["YL"], a["ZL"]), dtype=torch.float32, device=dev)
    obj = torch.as_tensor(np.ascontiguousarray(objects, dtype=np.float64).reshape(-1, 17), device=dev)
    st = torch.cuda.current_stream(dev)
    _lib.check(_lib.load().hr_project_ellipsoids(out.data_ptr(), a["YL"], a["ZL"], a["ViewN"], a["SO"], a["SD"],
                                                 a["dYA"], a["YLC0"], a["dZL"], a["ZLC0"], a["BetaS"], a["dBeta"],
                                                 a["h"], obj.data_ptr(), obj.shape[0], st.cuda_stream))
    st.synchronize()
    return out


def add_poisson_noise(proj: torch.Tensor, I0: float, seed: int) -> torch.Tensor:
    """In place: line integrals -> -log(max(N, 1)/I0), N ~ Poisson(I0 exp(-p)) (GPU)."""
    if not (proj.is_cuda and proj.dtype == torch.float32 and proj.is_contiguous()):
        raise TypeError("proj must be a contiguous CUDA float32 tensor")
    st = torch.cuda.current_stream(proj.device)
    _lib.check(_lib.load().hr_add_poisson_noise(proj.data_ptr(), proj.numel(), float(I0), int(seed) & ((1 << 64) - 1),
                                                st.cuda_stream))
    return proj
