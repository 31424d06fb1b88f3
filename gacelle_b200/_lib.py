"""ctypes binding of libgacelle_b200.so (include/gacelle_b200.h).

The library is built in-tree (``gacelle_b200/libgacelle_b200.so``) by
``gacelle_b200.build.build()``.  There is no CPU fallback: if the library is
missing, or no CUDA device is present, every compute call raises
:class:`GacelleError`.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgacelle_b200.so")

GX_OK, GX_EINVAL, GX_ENOMEM, GX_ECUDA, GX_EUNSUPPORTED, GX_ETIMEOUT, GX_ENUMERIC, GX_ECANCELLED = range(8)
STATUS_NAMES = {0: "ok", 1: "invalidArgument", 2: "outOfMemory", 3: "cuda", 4: "unsupported",
                5: "timeout", 6: "numeric", 7: "cancelled"}
MODEL_R2S, MODEL_R1R2S, MODEL_NEXI, MODEL_NEXI_RICE = 1, 2, 3, 4
LOSS = {"l1": 0, "l2": 1, "huber": 2, "mse": 3, "gauss": 4, "rician": 5}
OPTIMISER = {"adam": 0, "sgdm": 1, "rmsprop": 2}
TRANSFORM = {"sigmoid": 0, "linear": 1}
CONV_MODEL = {"ema": 0, "linear": 1}
PATH = {"fused": 0, "plain": 1}
REG_TV, REG_PRIOR, REG_SURFACE_TV = 0, 1, 2
STOP_REASONS = {0: "none", 1: "convergence", 2: "tol", 3: "step", 4: "grad"}
MEM_HOST, MEM_DEVICE = 0, 1

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)


class GacelleError(RuntimeError):
    """Error from the engine; ``identifier`` mirrors the reference's
    ``GACELLE:<...>`` error identifiers (``GACELLE:b200:<status>``)."""

    def __init__(self, status: int, message: str):
        self.status = status
        self.identifier = "GACELLE:b200:" + STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.identifier}: {message}")


class GxModel(C.Structure):
    _fields_ = [("kind", C.c_int32), ("lmax", C.c_int32), ("nx", C.c_int32),
                ("n_te", C.c_int32), ("te", _dp), ("n_fa", C.c_int32), ("fa_deg", _dp),
                ("tr", C.c_double), ("n_shell", C.c_int32), ("bval", _dp), ("big_delta", _dp)]


class GxVolume(C.Structure):
    _fields_ = [("dims", C.c_int32 * 3), ("nvox", C.c_int32), ("grid_index", _i32p),
                ("data", _fp), ("weights", _fp), ("theta0", _fp), ("b1", _fp), ("sigma", _fp),
                ("prior_mu", _fp), ("prior_sd", _fp), ("prior_offset", C.c_double),
                ("max_neighbours", C.c_int32), ("neighbours", _i32p), ("edge_length", _fp)]


class GxAskadamOpts(C.Structure):
    _fields_ = [("iteration", C.c_int32), ("initial_learn_rate", C.c_double),
                ("decay_rate", C.c_double), ("optimiser", C.c_int32), ("beta1", C.c_double),
                ("beta2", C.c_double), ("epsilon", C.c_double), ("momentum", C.c_double),
                ("rms_decay", C.c_double), ("rms_epsilon", C.c_double), ("loss", C.c_int32),
                ("mse_scale", C.c_double), ("huber_delta", C.c_double), ("sigma", C.c_double),
                ("transform", C.c_int32), ("randomness", C.c_double), ("seed", C.c_uint64),
                ("lb", _dp), ("ub", _dp), ("tol", C.c_double), ("convergence_value", C.c_double),
                ("convergence_window", C.c_int32), ("patience_convergence", C.c_double),
                ("convergence_model", C.c_int32), ("ema_decay", C.c_double),
                ("step_tol", C.c_double), ("grad_tol", C.c_double), ("patience_step", C.c_double),
                ("patience_grad", C.c_double), ("n_reg", C.c_int32), ("reg_param", C.c_int32 * 8),
                ("lambda_", C.c_double * 8), ("tv_3d", C.c_int32), ("voxel_size", C.c_double * 3),
                ("path", C.c_int32), ("chunk", C.c_int32), ("block_size", C.c_int32),
                ("robust_convergence", C.c_int32), ("outlier_weight", C.c_double),
                ("weight_update_interval", C.c_int32), ("outlier_check_window", C.c_int32),
                ("outlier_min_flag_duration", C.c_int32), ("outlier_voxel_thres", C.c_double),
                ("outlier_pop_thres", C.c_double), ("outlier_init_thres", C.c_double),
                ("outlier_init_pop_thres", C.c_double), ("reg_type", C.c_int32)]


class GxAskadamResult(C.Structure):
    _fields_ = [("final_theta", _fp), ("min_theta", _fp), ("final_residual", _fp),
                ("min_residual", _fp), ("final_resloss", _fp), ("min_resloss", _fp),
                ("loss_history", _dp), ("final_loss", C.c_double),
                ("final_loss_fidelity", C.c_double), ("final_loss_reg", C.c_double),
                ("min_loss", C.c_double), ("min_loss_fidelity", C.c_double),
                ("min_loss_reg", C.c_double), ("final_niteration", C.c_int32),
                ("min_niteration", C.c_int32), ("stop_reason", C.c_int32)]


class GxMcmcOpts(C.Structure):
    _fields_ = [("algorithm", C.c_int32), ("iteration", C.c_int32), ("thinning", C.c_int32),
                ("burnin", C.c_double), ("repetition", C.c_int32), ("nwalker", C.c_int32),
                ("step_size", C.c_double), ("start_range", C.c_double),
                ("ensemble_update", C.c_int32), ("x_step", _dp), ("lb", _dp), ("ub", _dp),
                ("seed", C.c_uint64), ("block_size", C.c_int32), ("is_global", _i32p),
                ("global_warmup", C.c_int32), ("nbin", C.c_int32)]


class GxMcmcResult(C.Structure):
    _fields_ = [("mean", _fp), ("std", _fp), ("posterior", _fp), ("n_accepted", C.c_int64),
                ("n_proposals", C.c_int64), ("ns", C.c_int32), ("n_global_accepted", C.c_int64),
                ("n_global_proposals", C.c_int64), ("median", _fp), ("iqr", _fp), ("mode", _fp)]


class GxTiming(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("main_kernel_ms", C.c_double),
                ("main_launches", C.c_int32), ("kernel_launches", C.c_int64),
                ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("tv_path", C.c_int32),
                ("block_size", C.c_int32), ("autotuned", C.c_int32), ("aux_kernel_ms", C.c_double)]


class GxTestHooks(C.Structure):
    _fields_ = [("fail_alloc_at", C.c_int32), ("wait_limit_cycles", C.c_int64),
                ("barrier_extra_arrivals", C.c_int32)]


TV_PERSISTENT, TV_PAIRS, TV_DATA_SMEM, TV_DATA_QUADS = 1, 2, 4, 8


STRUCTS = {"gx_model": GxModel, "gx_volume": GxVolume, "gx_askadam_opts": GxAskadamOpts,
           "gx_askadam_result": GxAskadamResult, "gx_mcmc_opts": GxMcmcOpts,
           "gx_mcmc_result": GxMcmcResult, "gx_timing": GxTiming, "gx_test_hooks": GxTestHooks}

# name -> (restype, argtypes) for every entry point declared in the header
SIGNATURES = {
    "gx_version": (C.c_char_p, []),
    "gx_abi_version": (C.c_int32, []),
    "gx_last_error": (C.c_char_p, []),
    "gx_struct_size": (C.c_size_t, [C.c_char_p]),
    "gx_context_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "gx_context_destroy": (C.c_int, [C.c_void_p]),
    "gx_context_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "gx_last_timing": (C.c_int, [C.c_void_p, C.POINTER(GxTiming)]),
    "gx_dictionary_match": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32,
                                      C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "gx_set_cancel_flag": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "gx_context_set_test_hooks": (C.c_int, [C.c_void_p, C.POINTER(GxTestHooks)]),
    "gx_model_sizes": (C.c_int, [C.POINTER(GxModel), _i32p, _i32p]),
    "gx_forward": (C.c_int, [C.c_void_p, C.POINTER(GxModel), C.c_int32, C.c_void_p, C.c_void_p,
                             C.c_int32, C.c_void_p]),
    "gx_model_gradient": (C.c_int, [C.c_void_p, C.POINTER(GxModel), C.c_int32, C.POINTER(GxVolume),
                                    C.POINTER(GxAskadamOpts), C.c_void_p, C.c_void_p, C.c_void_p,
                                    _dp, _dp, _dp]),
    "gx_askadam": (C.c_int, [C.c_void_p, C.POINTER(GxModel), C.c_int32, C.POINTER(GxVolume),
                             C.c_int32, C.POINTER(GxAskadamOpts), C.POINTER(GxAskadamResult)]),
    "gx_mcmc": (C.c_int, [C.c_void_p, C.POINTER(GxModel), C.c_int32, C.POINTER(GxVolume),
                          C.c_int32, C.POINTER(GxMcmcOpts), C.POINTER(GxMcmcResult)]),
    "gx_askadam_noalloc": (C.c_int, [C.POINTER(GxModel), C.c_void_p, C.c_void_p, C.c_int32,
                                     C.POINTER(GxAskadamOpts), C.c_void_p, C.c_void_p, _dp]),
}

_lib = None


def lib():
    """Load the engine library; raises GacelleError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GacelleError(GX_ECUDA, f"{LIB_PATH} is missing: build it with "
                                         "gacelle_b200.build.build() (there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int):
    if status != GX_OK:
        raise GacelleError(status, lib().gx_last_error().decode(errors="replace"))


class Context:
    """One engine context (device, stream, cached workspace)."""

    _default = {}

    def __init__(self, device: int = 0):
        self.ptr = C.c_void_p()
        check(lib().gx_context_create(device, C.byref(self.ptr)))
        self.device = device

    def close(self):
        if self.ptr:
            lib().gx_context_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        """Run this context's work on a CUDA stream given by its handle
        (``torch.cuda.Stream.cuda_stream``).  Handle 0, which is how PyTorch
        reports the default stream, selects the legacy default stream
        (cudaStreamLegacy); None returns to the context's own stream."""
        if stream_ptr is None:
            h = 0
        elif stream_ptr == 0:
            h = 1  # cudaStreamLegacy
        else:
            h = stream_ptr
        check(lib().gx_context_set_stream(self.ptr, C.c_void_p(h)))

    def timing(self) -> dict:
        t = GxTiming()
        check(lib().gx_last_timing(self.ptr, C.byref(t)))
        return {f: getattr(t, f) for f, _ in GxTiming._fields_}

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        if device not in cls._default:
            cls._default[device] = Context(device)
        return cls._default[device]
