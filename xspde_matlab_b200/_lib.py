"""ctypes binding of libxspde_b200.so (the C ABI declared in include/xspde_b200.h)."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libxspde_b200.so")

XS_OK = 0
ERRORS = {
    -1: "XS_ERR_SHAPE", -2: "XS_ERR_GRAMMAR", -3: "XS_ERR_NVRTC", -4: "XS_ERR_CUDA", -5: "XS_ERR_NAN",
    -6: "XS_ERR_TIMEOUT", -7: "XS_ERR_ARG", -8: "XS_ERR_NODEVICE", -9: "XS_ERR_UNSUPPORTED",
}
METHODS = {"MP": 0, "RK4": 1, "Euler": 2, "RK2": 3, "Implicit": 4}
MAXDIM = 4

# Every symbol include/xspde_b200.h declares.
EXPORTS = ["xs_create", "xs_destroy", "xs_last_error", "xs_version", "xs_observe_info", "xs_observe_shape",
           "xs_av_doubles_per_block",
           "xs_path_kind",
           "xs_run_path", "xs_run_path_device", "xs_sync", "xs_noise", "xs_random", "xs_step", "xs_compile_check",
           "xs_set_kernel_timing", "xs_kernel_stats", "xs_run_path_device_noalloc", "xs_noise_features",
           "xs_mlp_sizes", "xs_mlp_forward", "xs_mlp_train_grad", "xs_mlp_adam", "xs_batch_create",
           "xs_batch_destroy", "xs_batch_tune", "xs_batch_run", "xs_batch_sync", "xs_batch_av_doubles",
           "xs_batch_results", "xs_batch_info", "xs_set_boundary_values", "xs_run_path_raw", "xs_block_moments"]
KERNEL_KINDS = ["resident", "obs_reduce", "x_init", "x_step", "x_final", "y_pass", "x_obs", "scalar", "rc_pass"]


class XsProblem(ctypes.Structure):
    _fields_ = [
        ("dimensions", ctypes.c_int),
        ("fields", ctypes.c_int),
        ("noises", ctypes.c_int),
        ("inrandoms", ctypes.c_int),
        ("points", ctypes.c_int * MAXDIM),
        ("ranges", ctypes.c_double * MAXDIM),
        ("origins", ctypes.c_double * MAXDIM),
        ("steps", ctypes.c_int),
        ("checks", ctypes.c_int),
        ("ensembles", ctypes.c_int * 3),
        ("method", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("ipsteps", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("boundaries", ctypes.POINTER(ctypes.c_int)),
        ("deriv", ctypes.c_char_p),
        ("initial", ctypes.c_char_p),
        ("linear", ctypes.c_char_p),
        ("nobserve", ctypes.c_int),
        ("observe", ctypes.POINTER(ctypes.c_char_p)),
        ("nparams", ctypes.c_int),
        ("param_names", ctypes.POINTER(ctypes.c_char_p)),
        ("param_values", ctypes.POINTER(ctypes.c_double)),
        ("path_kind", ctypes.c_int),
        ("runtime_params", ctypes.c_int),
        ("transforms", ctypes.POINTER(ctypes.c_int)),
        ("sequence", ctypes.c_int),
        ("boundary_values", ctypes.c_int),
        ("knoises", ctypes.c_int),
        ("krandoms", ctypes.c_int),
        ("nfilter", ctypes.POINTER(ctypes.c_double)),
        ("rfilter", ctypes.POINTER(ctypes.c_double)),
        ("auxfields", ctypes.c_int),
        ("define", ctypes.c_char_p),
    ]


class XsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


_lib = None


def lib():
    """Load the in-tree library (built by xspde_matlab_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise OSError("libxspde_b200.so is not built; run xspde_matlab_b200/build.py")
        L = ctypes.CDLL(LIBPATH)
        P = ctypes.POINTER
        dp = P(ctypes.c_double)
        L.xs_create.argtypes = [P(XsProblem), P(ctypes.c_void_p)]
        L.xs_create.restype = ctypes.c_int
        L.xs_destroy.argtypes = [ctypes.c_void_p]
        L.xs_destroy.restype = None
        L.xs_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.xs_last_error.restype = ctypes.c_size_t
        L.xs_version.restype = ctypes.c_char_p
        L.xs_observe_info.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int)]
        L.xs_observe_info.restype = ctypes.c_int
        L.xs_observe_shape.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int)]
        L.xs_observe_shape.restype = ctypes.c_int
        L.xs_av_doubles_per_block.argtypes = [ctypes.c_void_p]
        L.xs_av_doubles_per_block.restype = ctypes.c_size_t
        L.xs_path_kind.argtypes = [ctypes.c_void_p]
        L.xs_path_kind.restype = ctypes.c_int
        L.xs_run_path.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
        L.xs_run_path.restype = ctypes.c_int
        L.xs_run_path_raw.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.xs_run_path_raw.restype = ctypes.c_int
        L.xs_run_path_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.xs_run_path_device.restype = ctypes.c_int
        L.xs_sync.argtypes = [ctypes.c_void_p]
        L.xs_sync.restype = ctypes.c_int
        L.xs_noise.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        L.xs_noise.restype = ctypes.c_int
        L.xs_random.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.xs_random.restype = ctypes.c_int
        L.xs_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.xs_step.restype = ctypes.c_int
        L.xs_compile_check.argtypes = [P(XsProblem), ctypes.c_char_p, ctypes.c_size_t]
        L.xs_compile_check.restype = ctypes.c_int
        L.xs_set_kernel_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.xs_set_kernel_timing.restype = ctypes.c_int
        L.xs_kernel_stats.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.xs_kernel_stats.restype = ctypes.c_int
        L.xs_run_path_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_void_p, ctypes.c_void_p]
        L.xs_run_path_device_noalloc.restype = ctypes.c_int
        L.xs_noise_features.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        L.xs_noise_features.restype = ctypes.c_int
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.xs_mlp_sizes.argtypes = [ci, ci, ci, P(ctypes.c_size_t)]
        L.xs_mlp_sizes.restype = ctypes.c_size_t
        L.xs_mlp_forward.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp]
        L.xs_mlp_forward.restype = ci
        L.xs_mlp_train_grad.argtypes = [ci, ci, ci, vp, vp, vp, vp, vp, vp, vp]
        L.xs_mlp_train_grad.restype = ci
        L.xs_mlp_adam.argtypes = [ctypes.c_size_t, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, ci, ctypes.c_float, vp]
        L.xs_mlp_adam.restype = ci
        L.xs_batch_create.argtypes = [vp, ci, P(vp)]
        L.xs_batch_create.restype = ci
        L.xs_batch_destroy.argtypes = [vp]
        L.xs_batch_destroy.restype = None
        L.xs_batch_tune.argtypes = [vp, ci]
        L.xs_batch_tune.restype = ci
        L.xs_batch_run.argtypes = [vp, vp]
        L.xs_batch_run.restype = ci
        L.xs_batch_sync.argtypes = [vp]
        L.xs_batch_sync.restype = ci
        L.xs_batch_av_doubles.argtypes = [vp, ci]
        L.xs_batch_av_doubles.restype = ctypes.c_size_t
        L.xs_batch_results.argtypes = [vp, ci, vp]
        L.xs_batch_results.restype = ci
        L.xs_batch_info.argtypes = [vp, ci, P(ci), ci]
        L.xs_batch_info.restype = ci
        L.xs_set_boundary_values.argtypes = [vp, ci, ci, vp]
        L.xs_set_boundary_values.restype = ci
        L.xs_block_moments.argtypes = [vp, ci, ctypes.c_longlong, ctypes.c_double, vp, ci, vp]
        L.xs_block_moments.restype = ci
        _ = dp
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(8192)
    lib().xs_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code):
    if code != XS_OK:
        raise XsError(code, last_error())
    return code
