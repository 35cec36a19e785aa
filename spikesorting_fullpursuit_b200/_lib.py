"""ctypes binding of libfbp_b200.so (the C ABI in include/fbp_b200.h).

There is no CPU fallback: if the library is missing or cannot be loaded,
`lib()` raises.  Error codes are mapped to the exceptions the reference
raises for the same conditions.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FBP_B200_LIB", os.path.join(_HERE, "libfbp_b200.so"))

FBP_OK = 0
FBP_ERR_BAD_ARG = 1
FBP_ERR_CUDA = 2
FBP_ERR_ITER_CAP = 3
FBP_ERR_CAPACITY = 4
FBP_ERR_NO_DEVICE = 5
FBP_ERR_OOM = 6
FBP_ERR_TIMEOUT = 7
DEFAULT_WAIT_POLLS = 16777216
NOALLOC_MAX_WINDOWS = 4194300
PREC_FP32 = 0
PREC_BF16_REFINE = 1
OVERLAP_FAST = 0
OVERLAP_EXACT = 1
TC_LAYOUT_AUTO = 0
TC_LAYOUT_SAMPLES = 1
TC_LAYOUT_WIDE = 2

_lib = None

U32 = ctypes.c_uint32
P = ctypes.c_void_p
SZ = ctypes.c_size_t
I = ctypes.c_int

F32, I16, F64 = 0, 1, 2
U64 = ctypes.c_uint64
I32 = ctypes.c_int32
I64 = ctypes.c_int64

# name -> (restype, argtypes); every symbol declared in include/fbp_b200.h
SIGNATURES = {
    "fbp_version": (I, []),
    "fbp_last_error": (ctypes.c_char_p, []),
    "fbp_pursuit_workspace_bytes": (I, [U32, U32, U32, U32, U32, I, ctypes.POINTER(SZ)]),
    "fbp_pursuit_chunk": (I, [P, U32, U32, P, U32, U32, P, P, U32, I, I, I, U32, P, SZ, P, P, U32, P,
                              ctypes.POINTER(U32), ctypes.POINTER(U32), I, P, P]),
    "fbp_compute_residual": (I, [P, U32, U32, P, U32, U32, P, P, U32, U32, P]),
    "fbp_get_adjusted_clips": (I, [P, U32, U32, P, U32, U32, P, P, U32, P, P]),
    "fbp_compute_full_likelihood": (I, [P, U32, U32, P, U32, U32, P, P, P, U32, P, I, P]),
    "fbp_window_argmax": (I, [U32, U32, U32, P, P, U32, P, P, P]),
    "fbp_overlap_recheck": (I, [P, U32, U32, P, U32, U32, P, P, U32, P, P, U32, P, P]),
    "fbp_check_overlap_reassignments": (I, [U32, U32, P, P, U32, P, P, P]),
    "fbp_binary_pursuit_accept": (I, [U32, U32, U32, P, P, P, U32, P, P, P, P, P, P, P, P, P, P]),
    "fbp_binary_pursuit_accept_noalloc": (I, [U32, U32, U32, P, P, P, U32, P, P, P, P, P, P, P, P]),
    "fbp_scan_scratch_bytes": (SZ, [U32]),
    "fbp_set_test_limits": (I, [P]),
    "fbp_set_tc_group_size": (I, [U32]),
    "fbp_set_tc_layout": (I, [I]),
    "fbp_tc_likelihood_bounds": (I, [P, U32, U32, P, U32, U32, P, P, SZ, P, P, P]),
    "fbp_window_u8_bytes": (SZ, [U32]),
}

# every symbol declared in include/fbp_prepost.h
PREPOST_SIGNATURES = {
    "fbp_get_clips": (I, [P, I, U64, U32, P, U32, P, U32, U32, I32, I32, P, P]),
    "fbp_robust_scratch_bytes": (SZ, [U32, U32, I]),
    "fbp_robust_templates": (I, [P, I, U32, U32, P, U32, P, P, SZ, P]),
    "fbp_noise_cov_scratch_bytes": (SZ, [U32, U32]),
    "fbp_clip_noise_covariance": (I, [P, I, P, P, P, U32, U32, U32, P, P, SZ, P]),
    "fbp_remove_duplicates": (I, [I, P, P, P, P, I, U32, P, U32, U32, I64, P, P, P]),
    "fbp_unit_mean_templates": (I, [P, U32, P, U32, P, P]),
    "fbp_overlap_template_scratch_bytes": (SZ, [U32, I32, I32]),
    "fbp_overlap_template_search": (I, [P, U32, U32, U32, I32, I32, P, U32, P, P, P, SZ, P]),
    "fbp_power_spectrum": (I, [P, I, U64, U64, P, P]),
    "fbp_wiener_smooth": (I, [P, I, U64, U64, I64, P, P]),
    "fbp_wiener_apply": (I, [P, P, P, I, U64, U64, P]),
    "fbp_zca_scratch_bytes": (SZ, [U32]),
    "fbp_zca_covariance": (I, [P, I, U32, U64, P, I32, P, P, P, SZ, P]),
    "fbp_zca_apply": (I, [P, P, I, U32, U64, P, P]),
    "fbp_separability_metrics": (I, [P, U32, U32, U32, P, ctypes.c_double, ctypes.c_double, P, P, P, P, P, P,
                                     P]),
}


N_STAGES = 9
STAGE_NAMES = ["likelihood", "argmax", "overlap", "check", "accept", "residual", "lists", "lik_refine",
               "overlap_tables"]


class StageStats(ctypes.Structure):
    """fbp_stage_stats of include/fbp_b200.h."""
    _fields_ = [("ms", ctypes.c_double * N_STAGES), ("launches", ctypes.c_uint64 * N_STAGES),
                ("work", ctypes.c_uint64 * N_STAGES), ("candidates", ctypes.c_uint64),
                ("refined_items", ctypes.c_uint64), ("fallback_candidates", ctypes.c_uint64),
                ("lik_refined", ctypes.c_uint64), ("lik_exact_passes", ctypes.c_uint64),
                ("passes", ctypes.c_uint32), ("spikes", ctypes.c_uint32),
                ("lik_lazy_refined", ctypes.c_uint64), ("lik_seq_refined", ctypes.c_uint64),
                ("tc_layout", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]

    def as_dict(self):
        return {"passes": self.passes, "spikes": self.spikes, "candidates": int(self.candidates),
                "refined_items": int(self.refined_items),
                "fallback_candidates": int(self.fallback_candidates),
                "lik_refined": int(self.lik_refined), "lik_exact_passes": int(self.lik_exact_passes),
                "lik_lazy_refined": int(self.lik_lazy_refined), "lik_seq_refined": int(self.lik_seq_refined),
                "tc_layout": {0: None, 1: "samples", 2: "wide"}.get(int(self.tc_layout)),
                "ms": {STAGE_NAMES[i]: self.ms[i] for i in range(N_STAGES)},
                "launches": {STAGE_NAMES[i]: int(self.launches[i]) for i in range(N_STAGES)},
                "work": {STAGE_NAMES[i]: int(self.work[i]) for i in range(N_STAGES)}}


class TestLimits(ctypes.Structure):
    """fbp_test_limits of include/fbp_b200.h."""
    _fields_ = [("refine_list_cap", ctypes.c_uint32), ("contender_pool_cap", ctypes.c_uint32),
                ("wait_polls", ctypes.c_uint32)]


def set_test_limits(refine_list_cap=0, contender_pool_cap=0, wait_polls=DEFAULT_WAIT_POLLS):
    """Testing hook: shrink the refinement list or contender pool, or shorten
    the tensor-core kernel's pipeline waits, for the calls that follow."""
    lim = TestLimits(int(refine_list_cap), int(contender_pool_cap), int(wait_polls))
    check(lib().fbp_set_test_limits(ctypes.byref(lim)))


def reset_test_limits():
    check(lib().fbp_set_test_limits(None))


class WindowState(ctypes.Structure):
    """fbp_window_state of include/fbp_b200.h."""
    _fields_ = [("best_idx", P), ("best_lab", P), ("best_ll", P), ("ov_idx", P),
                ("ov_lab", P), ("flags", P), ("overlap_recheck", P)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libfbp_b200.so not found at %s; build it with "
                "`python -m spikesorting_fullpursuit_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in list(SIGNATURES.items()) + list(PREPOST_SIGNATURES.items()):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class PursuitError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("fbp error %d: %s" % (code, msg))
        self.code = code


def check(rc):
    if rc == FBP_OK:
        return
    msg = lib().fbp_last_error().decode(errors="replace")
    if rc == FBP_ERR_BAD_ARG:
        raise ValueError(msg)
    raise PursuitError(rc, msg)


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream):
    return ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
