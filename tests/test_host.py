"""CPU tests of the host side: the C-ABI library's symbol table and struct
layouts, the layout helpers, the defaults restated from the reference, the
shell ordering of gpuNEXI, and the device header's Rician polynomial
coefficients (compiled for the host)."""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest
import scipy.special as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gacelle_b200.h")


@pytest.fixture(scope="module")
def lib():
    from gacelle_b200 import _lib, build
    build.build()
    return _lib.lib()


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gx_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point(lib):
    names = _declared_functions()
    assert len(names) >= 12
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "gacelle_b200", "libgacelle_b200.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (gx_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    from gacelle_b200 import _lib
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_struct_layouts_match_binding(lib):
    from gacelle_b200 import _lib
    for name, cls in _lib.STRUCTS.items():
        assert lib.gx_struct_size(name.encode()) == C.sizeof(cls), name
    assert lib.gx_struct_size(b"nope") == 0
    assert lib.gx_abi_version() == 6
    assert b"sm_100a" in lib.gx_version()


def test_no_device_is_a_loud_error(lib):
    """Without a usable CUDA device there is no CPU fallback: context creation fails."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gacelle_b200 import _lib
    ctx = C.c_void_p()
    st = lib.gx_context_create(0, C.byref(ctx))
    assert st == _lib.GX_ECUDA
    assert b"CUDA" in lib.gx_last_error() or b"device" in lib.gx_last_error()


def test_model_sizes_and_validation(lib):
    from gacelle_b200 import _lib
    from gacelle_b200.models import _GxModelHandle
    assert _GxModelHandle(_lib.MODEL_R2S, te=np.arange(12) * 1e-3).sizes() == (2, 12)
    assert _GxModelHandle(_lib.MODEL_R1R2S, te=np.arange(12) * 1e-3, fa_deg=[5, 20], tr=0.03).sizes() == (3, 24)
    b = np.ones(24)
    assert _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=b, lmax=0).sizes() == (4, 24)
    assert _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=b, lmax=2).sizes() == (5, 48)
    with pytest.raises(_lib.GacelleError) as e:
        _GxModelHandle(_lib.MODEL_NEXI, bval=b, delta=b, lmax=1).sizes()
    assert e.value.identifier == "GACELLE:b200:invalidArgument"
    with pytest.raises(_lib.GacelleError):
        _GxModelHandle(99).sizes()


def test_mask_index_is_column_major():
    from gacelle_b200 import utils
    m = np.zeros((3, 2, 2), bool)
    m[1, 0, 0] = m[0, 1, 0] = m[2, 1, 1] = True
    # MATLAB find() order: x fastest
    assert list(utils.mask_index(m)) == [1, 3, 11]


def test_nd_gd_round_trip():
    from gacelle_b200 import utils
    rng = np.random.default_rng(0)
    mask = rng.random((5, 4, 3)) > 0.4
    data = rng.normal(size=(5, 4, 3, 7))
    idx = utils.mask_index(mask)
    gd = utils.reshape_ND2GD(data, idx)
    assert gd.shape == (7, mask.sum()) and gd.flags["C_CONTIGUOUS"]
    back = utils.reshape_GD2ND(gd, mask)
    np.testing.assert_array_equal(back[mask], data[mask])
    assert np.all(back[~mask] == 0)


def test_askadam_defaults_match_reference():
    """askadam.check_set_default_basic (utils/askadam.m:735-878): the code's
    defaults (not the docstrings') are authoritative."""
    from gacelle_b200 import askadam_solver
    f = askadam_solver.check_set_default_basic({})
    assert f["lossFunction"] == "L1" and f["initialLearnRate"] == 0.001 and f["iteration"] == 1e4
    assert f["parameterTransform"] == "sigmoid" and f["convergenceModel"] == "ema"
    assert f["convergenceStepTol"] == 1e-6 and f["convergenceGradTol"] == 1e-6
    assert f["patienceConvergence"] == 5 and f["tol"] == 1e-3 and f["TVmode"] == "2D"
    assert f["voxelSize"] == [2, 2, 2] and f["adamupdateEpsilon"] == 1e-8
    g = askadam_solver.check_set_default_basic({"Nepoch": 77, "patience": 9})
    assert g["iteration"] == 77 and "Nepoch" not in g and g["patienceStep"] == 9


def test_mcmc_defaults_match_reference():
    from gacelle_b200 import mcmc_solver
    f = mcmc_solver.check_set_default_basic({"algorithm": "GW"})
    assert f["algorithm"] == "ensemble" and f["iteration"] == 2e5 and f["thinning"] == 20
    assert f["Nwalker"] == 50 and f["StepSize"] == 2 and f["startRange"] == 0.001
    assert f["Ensembleupdate"] == "simultaneous" and f["metric"] == ["mean", "std"]
    assert mcmc_solver.get_number_burnin({"iteration": 5000, "burnin": 0.2}) == 1000
    assert mcmc_solver.number_of_samples({"iteration": 5000, "burnin": 1000, "thinning": 10}) == 400


def test_nexi_shell_order_follows_constructor():
    """gpuNEXI sorts shells by DWIutility.unique_shell_keepb0: b = 0 dropped,
    Delta ascending, then b ascending (utils/DWIutility.m:735-772)."""
    from gacelle_b200 import gpuNEXI
    b = [6, 0, 1, 1, 6, 2.5]
    d = [49, 20, 49, 20, 20, 20]
    m = gpuNEXI(b, d)
    assert list(m.b) == [1, 2.5, 6, 1, 6] and list(m.Delta) == [20, 20, 20, 49, 49]


def test_update_property_strips_solver_parameters():
    from gacelle_b200 import gpuNEXI, gpuR2starMapping
    m = gpuNEXI([1, 2], [20, 20])
    m.updateProperty({"solver": "askadam", "lmax": 0})
    assert m.modelParams == ["fa", "Da", "De", "ra"] and len(m.lb) == 4
    m2 = gpuNEXI([1, 2], [20, 20])
    m2.updateProperty({"solver": "mcmc", "lmax": 2})
    assert m2.modelParams == ["fa", "Da", "De", "ra", "p2", "noise"]
    r = gpuR2starMapping([0.01])
    r.updateProperty({"solver": "askadam"})
    assert r.modelParams == ["M0", "R2star"] and r.startPoint == [1, 30]
    assert gpuR2starMapping([0.01]).modelParams[-1] == "noise"  # class contract untouched


def test_build_opts_maps_fitting(lib):
    from gacelle_b200 import askadam_solver
    f = askadam_solver.check_set_default_basic({"lossFunction": "MSE", "lambda": [1e-3], "regmap": ["R2star"],
                                               "TVmode": "3D", "patienceConvergence": float("inf")})
    o = askadam_solver.build_opts(f, ["M0", "R2star"], [0, 0.1], [2, 200])
    assert o.loss == 3 and o.n_reg == 1 and o.reg_param[0] == 1 and o.lambda_[0] == 1e-3 and o.tv_3d == 1
    assert o.patience_convergence == float("inf") and o.iteration == 10000
    with pytest.raises(Exception):
        askadam_solver.build_opts(dict(f, regmap=["nope"]), ["M0", "R2star"], [0, 0.1], [2, 200])


def test_custom_forward_functions_are_rejected():
    from gacelle_b200 import askadam, GacelleError
    with pytest.raises(GacelleError) as e:
        askadam().optimisation(np.ones((3, 4)), np.ones((1, 4)), None, {}, {}, lambda p: p)
    assert "unsupported" in e.value.identifier


def test_device_rician_polynomials_on_host(tmp_path):
    """The Abramowitz & Stegun 9.8.1-9.8.4 coefficients in gx_device.cuh,
    compiled for the host, against scipy's i0e / i1e."""
    src = tmp_path / "r.cpp"
    src.write_text('#include "gx_device.cuh"\n#include <cstdio>\nint main(){for(int i=0;i<=4000;++i){'
                   'float x=i*0.01f; float lg,omr; gx::rician_terms(x,lg,omr); printf("%.9g %.9g %.9g\\n",x,lg,omr);}}\n')
    exe = tmp_path / "r"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT}/gacelle_b200/csrc", "-I/usr/local/cuda/include",
                    str(src), "-o", str(exe)], check=True)
    out = np.loadtxt(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    x, lg, omr = out[:, 0], out[:, 1], out[:, 2]
    np.testing.assert_allclose(lg, np.log(sp.i0e(x)), atol=2e-6)
    ratio = sp.i1e(x) / sp.i0e(x)
    np.testing.assert_allclose(omr, 1 - ratio, rtol=5e-5, atol=5e-7)


def test_save_output_writes_a_mat_file(tmp_path):
    """askadam.save_askadam_output / mcmc.save_mcmc_output (utils/askadam.m:
    993-1009, utils/mcmc.m:702-718): the folder is created, the structure is
    the variable 'out'; an empty file name writes nothing."""
    import scipy.io
    from gacelle_b200.askadam_solver import askadam
    from gacelle_b200.mcmc_solver import mcmc
    out = {"final": {"M0": np.arange(6, dtype=np.float32).reshape(3, 2, 1), "loss": 0.25,
                     "stopReason": "convergence"},
           "lossHistory": np.linspace(1, 0, 5), "mask": np.ones((3, 2, 1), bool), "unused": None}
    p = tmp_path / "sub" / "fit.mat"
    assert askadam.save_askadam_output(str(p), out)
    m = scipy.io.loadmat(str(p), squeeze_me=True, struct_as_record=False)["out"]
    np.testing.assert_array_equal(m.final.M0, out["final"]["M0"][..., 0])
    assert m.final.loss == 0.25 and m.final.stopReason == "convergence"
    np.testing.assert_allclose(m.lossHistory, out["lossHistory"])
    assert not askadam.save_askadam_output([], out) and not mcmc.save_mcmc_output("", out)
    assert mcmc.save_mcmc_output(str(tmp_path / "m.mat"), {"mean": {"R2star": np.ones(4)}})


def test_r1r2s_true_flip_angle_becomes_b1():
    """extraData.trueFlipAngle (R1R2s/gpuJointR1R2starMapping.m:387-391),
    [x,y,z,1,Nfa] in radians: a per-voxel scale of the nominal angles becomes
    b1; a scale that differs between flip angles is rejected."""
    from gacelle_b200 import GacelleError, gpuJointR1R2starMapping
    m = gpuJointR1R2starMapping(np.linspace(2, 40, 12) * 1e-3, 0.03, [5.0, 20.0])
    b1 = np.random.default_rng(0).uniform(0.8, 1.2, (3, 4, 2))
    tfa = b1[..., None, None] * np.deg2rad([5.0, 20.0])
    ex = m._with_b1({"trueFlipAngle": tfa, "other": 1})
    np.testing.assert_allclose(ex["b1"], b1, rtol=1e-12)
    assert "trueFlipAngle" not in ex and ex["other"] == 1
    row = m._with_b1({"trueFlipAngle": b1.reshape(1, -1, 1) * np.deg2rad([5.0, 20.0])})
    np.testing.assert_allclose(row["b1"], b1.reshape(1, -1), rtol=1e-12)
    bad = tfa.copy()
    bad[0, 0, 0, 0, 1] *= 1.01
    with pytest.raises(GacelleError):
        m._with_b1({"trueFlipAngle": bad})
    with pytest.raises(GacelleError):
        m._with_b1({"trueFlipAngle": tfa[..., :1]})
    assert m._with_b1({"b1": b1})["b1"] is b1 and m._with_b1(None) is None


_MEX_API = """
/* Declarations of the MATLAB C matrix / MEX API functions the gateway uses,
   as documented by MathWorks (names and signatures only), for a compile check */
#include <stddef.h>
#include <stdbool.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxUNKNOWN_CLASS, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
               mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
               mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS } mxClassID;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
bool mxIsStruct(const mxArray*); bool mxIsEmpty(const mxArray*); bool mxIsChar(const mxArray*);
bool mxIsDouble(const mxArray*); bool mxIsSingle(const mxArray*); bool mxIsComplex(const mxArray*);
bool mxIsUint64(const mxArray*); bool mxIsInt32(const mxArray*); bool mxIsCell(const mxArray*);
mxArray* mxGetField(const mxArray*, mwIndex, const char*);
void mxSetField(mxArray*, mwIndex, const char*, mxArray*);
double mxGetScalar(const mxArray*); int mxGetString(const mxArray*, char*, mwSize);
size_t mxGetNumberOfElements(const mxArray*); size_t mxGetM(const mxArray*); size_t mxGetN(const mxArray*);
double* mxGetPr(const mxArray*); void* mxGetData(const mxArray*); mxArray* mxGetCell(const mxArray*, mwIndex);
mxArray* mxCreateNumericMatrix(mwSize, mwSize, mxClassID, mxComplexity);
mxArray* mxCreateDoubleMatrix(mwSize, mwSize, mxComplexity); mxArray* mxCreateDoubleScalar(double);
mxArray* mxCreateStructMatrix(mwSize, mwSize, int, const char**); void mxDestroyArray(mxArray*);
void mexErrMsgIdAndTxt(const char*, const char*, ...); void mexWarnMsgIdAndTxt(const char*, const char*, ...);
"""


def test_mex_gateway_compiles_against_the_mex_api(tmp_path):
    """The MATLAB gateway (gacelle_b200/matlab/gacelle_b200_mex.c) is built only
    where MATLAB is installed; here it is compiled against declarations of the
    documented MEX API functions it calls and the C-ABI header, with warnings
    as errors, so that a signature it passes to the engine cannot drift."""
    (tmp_path / "mex.h").write_text(_MEX_API)
    src = os.path.join(ROOT, "gacelle_b200", "matlab", "gacelle_b200_mex.c")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
                        "-I", str(tmp_path), "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
