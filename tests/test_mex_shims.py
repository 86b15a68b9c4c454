"""The mexFunction shims (analyticalreconbigpatient_b200/mex/*.cpp) built as MEX-style
shared libraries against an in-process stand-in for MATLAB's mx runtime
(tests/mexfake), then called the way MATLAB calls them: argument checks on the
CPU; on the GPU, results identical to the C-ABI calls the shims wrap."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "analyticalreconbigpatient_b200")
SHIMS = ("ParallelRebinningCBCurve", "reWeigAdFiltr_GPU", "Parallel_FDK_Helical_3DWeighting")
DOUBLE, SINGLE, INT32 = 6, 7, 12
CLASS = {np.float64: DOUBLE, np.float32: SINGLE, np.int32: INT32}


class MexError(Exception):
    pass


class Mex:
    """One shim linked with the fake runtime; call(nlhs, *args) like MATLAB."""

    def __init__(self, so: str):
        self.lib = ctypes.CDLL(so, mode=ctypes.RTLD_LOCAL)
        L = self.lib
        L.mxf_wrap.restype = ctypes.c_void_p
        L.mxf_wrap.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]
        L.mxf_struct.restype = ctypes.c_void_p
        L.mxf_struct.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.mxf_data.restype = ctypes.c_void_p
        L.mxf_data.argtypes = [ctypes.c_void_p]
        L.mxf_numel.restype = ctypes.c_longlong
        L.mxf_numel.argtypes = [ctypes.c_void_p]
        L.mxf_free.argtypes = [ctypes.c_void_p]
        L.mxf_call.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                               ctypes.POINTER(ctypes.c_void_p)]
        L.mxf_error.restype = ctypes.c_char_p
        self._keep = []

    def array(self, a: np.ndarray):
        """A C-order numpy array as the MATLAB array with the reversed dims (no copy)."""
        a = np.ascontiguousarray(a)
        self._keep.append(a)
        dims = (ctypes.c_longlong * max(a.ndim, 1))(*(reversed(a.shape) if a.ndim else (1,)))
        return self.lib.mxf_wrap(CLASS[a.dtype.type], max(a.ndim, 1), dims, a.ctypes.data)

    def struct(self, *fields):
        ptrs = (ctypes.c_void_p * len(fields))(*fields)
        return self.lib.mxf_struct(len(fields), ptrs)

    def call(self, nlhs: int, *args):
        prhs = (ctypes.c_void_p * max(len(args), 1))(*args)
        plhs = (ctypes.c_void_p * max(nlhs, 1))()
        if self.lib.mxf_call(nlhs, plhs, len(args), prhs):
            raise MexError(self.lib.mxf_error().decode())
        outs = []
        for k in range(nlhs):
            n = self.lib.mxf_numel(plhs[k])
            outs.append(np.ctypeslib.as_array((ctypes.c_float * n).from_address(self.lib.mxf_data(plhs[k]))).copy())
            self.lib.mxf_free(plhs[k])
        return outs


@pytest.fixture(scope="session")
def mex(tmp_path_factory):
    """Builds each shim + the fake runtime into its own shared library (as `mex` would)."""
    if not os.path.exists(os.path.join(PKG, "libhelixrecon.so")):
        pytest.fail("libhelixrecon.so is not built")
    out = tmp_path_factory.mktemp("mex")
    libs = {}
    for name in SHIMS:
        so = str(out / f"{name}.so")
        subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-Wall", "-Werror",
                        "-I", os.path.join(ROOT, "tests", "mexfake"), "-I", os.path.join(ROOT, "include"),
                        os.path.join(PKG, "mex", f"{name}.cpp"), os.path.join(ROOT, "tests", "mexfake", "mexfake.cpp"),
                        "-L", PKG, "-lhelixrecon", f"-Wl,-rpath,{PKG}", "-o", so], check=True)
        libs[name] = Mex(so)
    return libs


def s(v):
    return np.array([v], np.float32)


def i(v):
    return np.array([v], np.int32)


def scan_geom(m: Mex, sc, ObjR, obj_centre):
    d = lambda v: m.array(np.asarray(v, np.float64))
    return m.struct(d([sc.SO, sc.DO, sc.YL, sc.ZL, sc.DecWidth, sc.DecHeigh, 0.0, sc.ZLC1, sc.h_norm]),
                    d([sc.bp_geom()["BetaS"], 0.0, sc.PN, sc.N_2pi]),
                    d([ObjR, sc.XN, sc.YN, sc.ZN, *obj_centre]),
                    d([sc.delta, sc.HSCoef, sc.mk1]))


def test_shims_reject_bad_arguments_before_any_device_work(mex):
    r = mex["ParallelRebinningCBCurve"]
    proj = np.zeros((4, 8, 2), np.float32)
    good = [proj, i(8), i(2), i(4), s(4.5), s(0.01), s(0.1), s(4.5), s(1.0), s(0.1), s(541.0), i(1)]
    with pytest.raises(MexError, match="helixrecon:ParallelRebinningCBCurve: .*12 inputs"):
        r.call(1, *[r.array(a) for a in good[:11]])
    bad = list(good)
    bad[1] = np.array([8.0])  # double where the driver passes int32(YL)
    with pytest.raises(MexError, match="YL must be int32"):
        r.call(1, *[r.array(a) for a in bad])
    bad = list(good)
    bad[0] = np.zeros((4, 8, 1), np.float32)  # too few samples for ZL*YL*ViewN
    with pytest.raises(MexError, match="Proj must be single"):
        r.call(1, *[r.array(a) for a in bad])
    f = mex["reWeigAdFiltr_GPU"]
    fargs = [f.array(a) for a in (np.zeros((3, 2, 8), np.float32), s(3.5), s(0.5), s(1.0), s(1.0), s(541.0))]
    with pytest.raises(MexError, match="6 inputs and gives one output"):
        f.call(0, *fargs)
    with pytest.raises(MexError, match="dZL must be single"):
        f.call(1, *fargs[:4], f.array(np.array([1.0])), fargs[5])
    b = mex["Parallel_FDK_Helical_3DWeighting"]
    geom = b.struct(*[b.array(np.zeros(n)) for n in (9, 4, 6, 3)])  # Obj one short
    bargs = [geom, b.array(np.zeros(8)), b.array(np.zeros(8)), b.array(i(1))]
    with pytest.raises(MexError, match="does not need any output"):
        b.call(1, *bargs)
    with pytest.raises(MexError, match="ScanGeom.Obj must hold 7 doubles"):
        b.call(0, *bargs)
    with pytest.raises(MexError, match="needs 4 inputs"):
        b.call(0, *bargs[:3])


@pytest.mark.gpu
def test_rebin_shim_matches_c_abi_and_reference(mex, cuda):
    import oracle
    from analyticalreconbigpatient_b200 import api, geometry as G

    sc = G.tiny(ZL=6, YL=200, det_pitch=1.0239 * 888 / 200, iso_channel=100.75)
    ra = sc.rebin_args()
    proj = np.random.default_rng(3).random((ra["ViewN"], ra["YL"], ra["ZL"]), dtype=np.float32)
    m = mex["ParallelRebinningCBCurve"]
    args = [proj, i(ra["YL"]), i(ra["ZL"]), i(ra["ViewN"]), s(ra["YLC"] + 1), s(ra["dYA"]), s(ra["DeltaTheta"]),
            s(ra["PLC"] + 1), s(ra["DeltaT"]), s(ra["DeltaFai"]), s(ra["SO"]), i(1)]
    (out,) = m.call(1, *[m.array(a) for a in args])
    mine = api.ParallelRebinningCBCurve(proj, ra["YL"], ra["ZL"], ra["ViewN"], ra["YLC"] + 1, ra["dYA"],
                                        ra["DeltaTheta"], ra["PLC"] + 1, ra["DeltaT"], ra["DeltaFai"], ra["SO"], 1)
    np.testing.assert_array_equal(out.view(np.uint32), mine.ravel().view(np.uint32))
    ref = oracle.rebin_f32(proj, **ra)
    np.testing.assert_array_equal(out.view(np.uint32), ref.ravel().view(np.uint32))


@pytest.mark.gpu
def test_filter_shim_matches_c_abi(mex, cuda):
    from analyticalreconbigpatient_b200 import api, geometry as G

    fa = G.tiny(YL=150, ZL=7).filter_args()
    p = np.random.default_rng(5).standard_normal((40, fa["ZL"], fa["YL"])).astype(np.float32)
    m = mex["reWeigAdFiltr_GPU"]
    (out,) = m.call(1, *[m.array(a) for a in (p, s(fa["PLC"]), s(fa["ZLC"]), s(fa["dYL"]), s(fa["dZL"]),
                                              s(fa["SO"]))])
    mine = api.reWeigAdFiltr_GPU(p, fa["PLC"], fa["ZLC"], fa["dYL"], fa["dZL"], fa["SO"])
    np.testing.assert_array_equal(out.view(np.uint32), mine.ravel().view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("use_gpu", [0, 1])
def test_backprojection_shim_writes_ctimage_in_place(mex, cuda, use_gpu):
    from analyticalreconbigpatient_b200 import api, geometry as G

    # the MEX derives cubic voxels dx = dy = dz = 2 ObjR / N: a 6 mm cube of 0.5 mm voxels inside the helix
    sc = G.tiny(delta=8, XN=12, YN=12, ZN=12, dx=0.5, dy=0.5, dz=0.5)
    ObjR = sc.dx * sc.XN / 2
    g = sc.bp_geom()
    centre = [g["XNC"] + 1, g["YNC"] + 1, g["ZNC"] + 1]
    fp = np.random.default_rng(9).standard_normal((g["PN"], g["ZL"], g["YL"]))
    m = mex["Parallel_FDK_Helical_3DWeighting"]
    ct = np.zeros(sc.XN * sc.YN * sc.ZN)
    m.call(0, scan_geom(m, sc, ObjR, centre), m.array(fp), m.array(ct), m.array(i(use_gpu)))
    ref = np.zeros_like(ct)
    api.Parallel_FDK_Helical_3DWeighting(
        {"ScDet": [sc.SO, sc.DO, sc.YL, sc.ZL, sc.DecWidth, sc.DecHeigh, 0.0, sc.ZLC1, sc.h_norm],
         "Proj": [g["BetaS"], 0.0, sc.PN, sc.N_2pi], "Obj": [ObjR, sc.XN, sc.YN, sc.ZN, *centre],
         "Rec": [sc.delta, sc.HSCoef, sc.mk1]}, fp, ref, use_gpu)
    assert np.count_nonzero(ct) > ct.size // 4
    np.testing.assert_array_equal(ct, ref)
