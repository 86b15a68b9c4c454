"""Scan and reconstruction-grid geometry.

Restates the scalar derivations the reference's MATLAB driver performs before
each of its three MEX calls, so that callers need no MATLAB:

* scanner/helix scalars        src/analyticalReconBigPatient.m:35-75
* rebinning arguments          src/Parallel_Rebinning_CB_Curve.m:8-18
* segment overlap (half fan)   src/analyticalRecon.m:15-16
* post-rebin crop              src/analyticalReconBigPatient.m:80-93
* filter arguments             src/analyticalReconBigPatient.m:95-105,139
* backprojection scalars       src/Parallel_FDK_Helical_3DWeighting.cpp:145-170,222-263

Conventions (all fixed by the reference's formulas):

* Fan view ``i`` has source angle ``BetaS + i*2*pi/N_2pi`` and source height
  ``h*angle/(2*pi)`` (absolute angle, ``..._3DWeighting.cpp:62,79``).
* Channel indices are the post-flip ones (``analyticalReconBigPatient.m:30-31``):
  fan angle ``(j - YLC0)*dYA``.
* Rebinned parallel view ``p`` is backprojected at ``BetaS_bp + p*2*pi/N_2pi``.
* Volume index ``(xi, yi, zi)`` sits at ``((xi-XNC)dx, (yi-YNC)dy, (zi-ZNC)dz)``,
  stored ``[YN][XN][ZN]`` with z fastest.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

TWO_PI = 2.0 * math.pi
# The reference's file-level pi (src/Parallel_FDK_Helical_3DWeighting.cpp:16),
# used by its CPU backprojection for the central view s0 (:62).
PI_TRUNC = 3.14159265358979
MU_WATER = 0.0193  # 1/mm


@dataclass(frozen=True)
class Scan:
    """One helical scan on a curved (arc) detector plus its output grid."""

    # scanner
    SO: float = 541.0            # source to isocentre (mm)
    SD: float = 949.0            # source to detector (mm)
    YL: int = 888                # channels per row
    det_pitch: float = 1.0239    # channel pitch at the detector surface (mm)
    ZL: int = 16                 # detector rows
    row_height: float = 1.0963   # row height at the detector surface (mm)
    N_2pi: int = 984             # views per rotation
    pitch: float = 0.9375        # table feed per rotation / (ZL * row height at iso)
    rotations: float = 4.0
    iso_channel: float | None = None  # YLC, 1-based, after the channel flip; default (YL+1)/2
    beta_start: float | None = None   # source angle of fan view 0; default centres the scan on z = 0
    # reconstruction
    XN: int = 256
    YN: int = 256
    ZN: int = 32
    dx: float = 1.5625
    dy: float = 1.5625
    dz: float = 1.0
    z_centre: float = 0.0        # z (mm) of the grid centre
    delta: int = 60              # taper length of the view weight (views)
    HSCoef: float = 0.68         # half-scan coefficient
    mk1: float = 5.0             # 3D-weight exponent before scaling by the pitch
    crop_both_ends: bool = True  # drop the half-fan margin at both scan ends after rebinning

    # ---------------------------------------------------------------- scanner
    @property
    def DO(self) -> float:
        return self.SD - self.SO

    @property
    def views(self) -> int:
        return int(round(self.rotations * self.N_2pi))

    @property
    def DecAngle(self) -> float:  # m-file :45
        return math.atan(self.det_pitch / self.SD / 2.0) * self.YL * 2.0

    @property
    def dYA(self) -> float:  # Parallel_Rebinning_CB_Curve.m:11
        return self.DecAngle / self.YL

    @property
    def DecHeigh(self) -> float:  # m-file :46
        return self.row_height * self.ZL

    @property
    def h_norm(self) -> float:
        """ScDet(9): pitch relative to the detector height at the detector."""
        return self.pitch * self.SO / self.SD  # m-file :48 with HelicalPitch = pitch * ZL

    @property
    def h(self) -> float:
        """Table feed per rotation (mm), as the MEX forms it: ScDet(9)*DecHeigh."""
        return self.h_norm * self.DecHeigh

    @property
    def k1(self) -> float:  # ..._3DWeighting.cpp:250
        return self.mk1 * self.h_norm

    @property
    def YLC1(self) -> float:
        return (self.YL + 1) * 0.5 if self.iso_channel is None else float(self.iso_channel)

    @property
    def ZLC1(self) -> float:  # m-file :40
        return (1 + self.ZL) * 0.5

    @property
    def dBeta(self) -> float:
        return TWO_PI / self.N_2pi

    @property
    def BetaS(self) -> float:
        if self.beta_start is not None:
            return float(self.beta_start)
        return -(self.views - 1) * 0.5 * self.dBeta

    @property
    def seg_overlap(self) -> int:  # analyticalRecon.m:15-16
        so = math.atan(self.det_pitch / self.SD / 2.0) * self.YL
        return int(math.ceil(so * self.N_2pi / TWO_PI)) + 1

    # ---------------------------------------------------------------- rebin
    def rebin_args(self) -> dict:
        """Arguments of the C entry ParallelRebinningCBCurve_GPU (0-based YLC/PLC),
        float32-rounded as the MEX passes them (Parallel_Rebinning_CB_Curve.m:8-18,
        ParallelRebinningCBCurve.cpp:119-128)."""
        ViewN = self.views
        BetaE = self.BetaS + ViewN * self.dBeta  # m-file :70
        DeltaFai = (BetaE - self.BetaS) / (ViewN - 1)
        DeltaT = math.tan(self.DecAngle * 0.5) * self.SO * 1.5 * 2.0 / self.YL
        PLC1 = (1 + self.YL) * 0.5
        f = np.float32
        return dict(YL=self.YL, ZL=self.ZL, ViewN=ViewN, YLC=float(f(self.YLC1) - f(1.0)), dYA=float(f(self.dYA)),
                    DeltaTheta=float(f(DeltaFai)), PLC=float(f(PLC1) - f(1.0)), DeltaT=float(f(DeltaT)),
                    DeltaFai=float(f(DeltaFai)), SO=float(f(self.SO)))

    # ---------------------------------------------------------------- crop
    @property
    def crop_front(self) -> int:
        return self.seg_overlap if self.crop_both_ends else 0

    @property
    def crop_back(self) -> int:
        return self.seg_overlap

    @property
    def PN(self) -> int:
        return self.views - self.crop_front - self.crop_back

    @property
    def BetaS_bp(self) -> float:  # m-file :87
        return self.BetaS + self.crop_front * self.dBeta

    # ---------------------------------------------------------------- filter
    @property
    def DecWidth(self) -> float:  # m-file :95
        return math.tan(self.DecAngle * 0.5) * self.SO * 2.0 * 1.5

    @property
    def dYL(self) -> float:
        return self.DecWidth / self.YL

    @property
    def dZL(self) -> float:
        return self.DecHeigh / self.ZL

    def filter_args(self) -> dict:
        """Arguments of the C entry `filtering` (m-file :139: PLC-1, ZLC-1, float32)."""
        f = np.float32
        PLC1 = (1 + self.YL) * 0.5
        return dict(YL=self.YL, ZL=self.ZL, ViewN=self.PN, PLC=float(f(PLC1 - 1.0)), ZLC=float(f(self.ZLC1 - 1.0)),
                    dYL=float(f(self.dYL)), dZL=float(f(self.dZL)), SO=float(f(self.SO)))

    # ---------------------------------------------------------------- backprojection
    @property
    def XNC(self) -> float:
        return (self.XN - 1) * 0.5

    @property
    def YNC(self) -> float:
        return (self.YN - 1) * 0.5

    @property
    def ZNC(self) -> float:
        return (self.ZN - 1) * 0.5 - self.z_centre / self.dz

    def bp_geom(self) -> dict:
        """Scalars of ParallekFDKHelical3DWeighting_GPU_{float,double} in double,
        as ParallelFDKHelical3DWeighting derives them (..._3DWeighting.cpp:145-154),
        with explicit (possibly anisotropic) dx, dy, dz. YLC is (YL-1)/2 as the MEX
        forces it (:229)."""
        return dict(N_2pi=self.N_2pi, XN=self.XN, YN=self.YN, ZN=self.ZN, XNC=self.XNC, YNC=self.YNC, ZNC=self.ZNC,
                    dx=self.dx, dy=self.dy, dz=self.dz, YL=self.YL, ZL=self.ZL, PN=self.PN,
                    YLC=(self.YL - 1) * 0.5, ZLC=self.ZLC1 - 1.0, dYL=self.dYL, dZL=self.dZL, h=self.h,
                    BetaS=self.BetaS_bp, DeltaFai=2.0 * 3.141592653589793 / self.N_2pi, N_pi=self.N_2pi / 2.0,
                    HSCoef=self.HSCoef, SO=self.SO, SD=self.SO + self.DO, k1=self.k1)

    # ---------------------------------------------------------------- accounting
    def window_per_slice(self) -> np.ndarray:
        """Clamped [s1, s2] view count per z slice, with the backprojection's own
        central-view rule (..._3DWeighting.cpp:61-70)."""
        g = self.bp_geom()
        zi = np.arange(self.ZN, dtype=np.float64)
        z = (zi - g["ZNC"]) * g["dz"]
        beta0 = 2.0 * PI_TRUNC * z / g["h"]
        s0 = np.ceil((beta0 - g["BetaS"]) / g["DeltaFai"] - 0.5)
        half = math.ceil(g["N_pi"] * g["HSCoef"])
        s1 = s0 - half
        s2 = s0 + half
        ok = (s1 < g["PN"]) & (s2 > 0)
        s1c = np.maximum(s1, 0)
        s2c = np.minimum(s2, g["PN"] - 1)
        return np.where(ok, s2c - s1c + 1, 0).astype(np.int64)

    def updates(self) -> int:
        """Voxel-view updates: every (voxel, view) pair in the clamped window."""
        return int(self.window_per_slice().sum()) * self.XN * self.YN

    def fully_sampled_slices(self) -> int:
        half = math.ceil(self.N_2pi / 2.0 * self.HSCoef)
        span = self.h * (self.PN - 2 * half) / self.N_2pi
        return max(1, int(math.floor(span / self.dz)))

    def with_full_z(self) -> "Scan":
        """The same scan with ZN spanning the fully sampled z range."""
        return replace(self, ZN=self.fully_sampled_slices())

    def projection_bytes(self) -> int:
        return 4 * self.YL * self.ZL * self.views

    def volume_bytes(self) -> int:
        return 4 * self.XN * self.YN * self.ZN


def config(name: str) -> Scan:
    """Workloads of the benchmark configurations, by name.

    small    888x16 curved detector, 984 views/rot, pitch 0.9375, 4 rotations,
             256x256x32 at 1.5625 x 1.5625 x 1.0 mm (Shepp-Logan head phantom)
    full     888x64, pitch 0.984, 20 rotations, 512x512xN at 0.9766 x 0.625 mm,
             N spanning the fully sampled z range (random ellipsoid phantom)
    halfview full geometry at 492 views/rot and 10 rotations
    bigpatient full detector, 200 rotations (196,800 views, 44.7 GB), 512x512x2000
             with the slice thickness chosen so the 2000 slices span the fully
             sampled z range (3.92 mm)
    """
    if name == "small":
        return Scan(ZL=16, pitch=0.9375, rotations=4, XN=256, YN=256, ZN=32, dx=1.5625, dy=1.5625, dz=1.0)
    if name == "full":
        return Scan(ZL=64, pitch=0.984, rotations=20, XN=512, YN=512, ZN=1, dx=0.9766, dy=0.9766,
                    dz=0.625).with_full_z()
    if name == "medium":  # full detector and grid spacing, 2 rotations: a profiling-size case
        return Scan(ZL=64, pitch=0.984, rotations=2, XN=512, YN=512, ZN=48, dx=0.9766, dy=0.9766, dz=0.625)
    if name == "bigpatient":  # 200 rotations; 2000 slices spanning the fully sampled z range
        sc = Scan(ZL=64, pitch=0.984, rotations=200, XN=512, YN=512, ZN=2000, dx=0.9766, dy=0.9766, dz=1.0)
        half = math.ceil(sc.N_2pi / 2.0 * sc.HSCoef)
        return replace(sc, dz=sc.h * (sc.PN - 2 * half) / sc.N_2pi / sc.ZN)
    if name == "halfview":
        return Scan(ZL=64, pitch=0.984, rotations=10, N_2pi=492, XN=512, YN=512, ZN=1, dx=0.9766, dy=0.9766,
                    dz=0.625).with_full_z()
    raise KeyError(name)


def batch_scans(seed: int = 6, n: int = 12) -> list[Scan]:
    """The uneven batch: ``n`` independent scans on the 888-channel detector at
    984 views/rotation with rotations uniform in 2..30, rows from {16, 32, 64},
    pitch from {0.5, 0.9375, 1.375} and a 256x256 (1.953 mm) or 512x512
    (0.9766 mm) grid of 32..400 slices, drawn from a seeded SplitMix64 stream.
    Slices are 0.625 mm thick, or thinner where the fully sampled z range of a
    short scan is shorter than the drawn slice count at 0.625 mm, so every
    slice lies in the fully sampled range."""
    from .phantom import SplitMix64

    rng = SplitMix64(seed)
    pick = lambda opts: opts[min(int(rng.uniform() * len(opts)), len(opts) - 1)]
    out = []
    for _ in range(n):
        rot = min(2 + int(rng.uniform() * 29), 30)
        ZL = pick((16, 32, 64))
        pitch = pick((0.5, 0.9375, 1.375))
        N = pick((256, 512))
        ZN = min(32 + int(rng.uniform() * 369), 400)
        d = 500.0 / N
        sc = Scan(ZL=ZL, pitch=pitch, rotations=rot, XN=N, YN=N, ZN=ZN, dx=d, dy=d, dz=0.625)
        half = math.ceil(sc.N_2pi / 2.0 * sc.HSCoef)
        span = sc.h * (sc.PN - 2 * half) / sc.N_2pi
        out.append(replace(sc, dz=min(0.625, span / ZN)))
    return out


def tiny(**kw) -> Scan:
    """A scaled-down scan for CPU-speed tests: same detector geometry family with
    fewer channels, rows and views."""
    base = dict(SO=541.0, SD=949.0, YL=96, ZL=8, row_height=1.0963, N_2pi=120, pitch=0.9375, rotations=3, XN=24,
                YN=24, ZN=6, dx=12.0, dy=12.0, dz=1.5)
    base.update(kw)
    base.setdefault("det_pitch", 1.0239 * 888 / base["YL"])  # keep the full detector's fan angle
    return Scan(**base)
