"""ctypes binding of the fftcorr_b200 C ABI (include/fc_api.h).

The shared library is built in-tree (``python -m fftcorr_b200._build``).  There
is no CPU fallback: every call below runs on the GPU, and a missing library or
device raises immediately.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfftcorr_b200.so")

FC_OK = 0
FC_ERR_INVALID = -1
FC_ERR_RANGE = -2
FC_ERR_ALLOC = -3
FC_ERR_CUDA = -4
FC_ERR_CUFFT = -5
FC_ERR_STATE = -6
FC_ERR_UNSUPPORTED = -7
FC_ERR_TIMEOUT = -8
FC_ERR_ADMISSION = -9
FC_FAULT_DEVICE_ALLOC = 1
FC_FAULT_FFT_PLAN = 2

FC_FP64 = 0
FC_FP32_MIXED = 1
FC_PERIODIC = 0
FC_SURVEY = 1

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)


class FcError(RuntimeError):
    """A CUDA, cuFFT or call-order failure reported by the library."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class AdmissionError(FcError):
    pass


class AssignStats(ctypes.Structure):
    _fields_ = [("num_added", ctypes.c_uint64), ("num_skipped", ctypes.c_uint64),
                ("totw", ctypes.c_double), ("totwsq", ctypes.c_double),
                ("sort_time", ctypes.c_double), ("window_time", ctypes.c_double)]


class CorrTimings(ctypes.Structure):
    _fields_ = [("total_time", ctypes.c_double), ("fft_time", ctypes.c_double),
                ("ylm_time", ctypes.c_double), ("multiply_time", ctypes.c_double),
                ("extract_time", ctypes.c_double),
                ("histogram_time", ctypes.c_double),
                ("setup_time", ctypes.c_double), ("n_fft", ctypes.c_int)]


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int),
                ("seconds", ctypes.c_double)]


class BatchBox(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int * 3), ("cell_size", ctypes.c_double),
                ("posw_device", ctypes.c_void_p), ("n", ctypes.c_int64)]


class BatchParams(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int), ("window", ctypes.c_int),
                ("rmax", ctypes.c_double), ("dr", ctypes.c_double),
                ("kmax", ctypes.c_double), ("dk", ctypes.c_double),
                ("maxell", ctypes.c_int), ("precision", ctypes.c_int),
                ("lanes", ctypes.c_int), ("tune", ctypes.c_int)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("nboxes", ctypes.c_int), ("lanes", ctypes.c_int),
                ("hist_blocks", ctypes.c_int), ("graph_nodes", ctypes.c_int64),
                ("kernel_nodes", ctypes.c_int64), ("own_kernel_nodes", ctypes.c_int64),
                ("hist_items", ctypes.c_int64), ("device_bytes", ctypes.c_int64)]


class CatalogSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n", ctypes.c_int64),
                ("posw", ctypes.c_void_p), ("boxsize", ctypes.c_double),
                ("ncentres", ctypes.c_int), ("sigma", ctypes.c_double),
                ("rmin", ctypes.c_double), ("rmax", ctypes.c_double),
                ("ra_half", ctypes.c_double), ("dec_half", ctypes.c_double),
                ("wmin", ctypes.c_double), ("wmax", ctypes.c_double),
                ("wsign", ctypes.c_double), ("seed", ctypes.c_uint64)]


class Job(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("shape", ctypes.c_int * 3),
                ("cell", ctypes.c_double), ("posmin", ctypes.c_double * 3),
                ("scheme", ctypes.c_int), ("window", ctypes.c_int),
                ("rmax", ctypes.c_double), ("dr", ctypes.c_double),
                ("kmax", ctypes.c_double), ("dk", ctypes.c_double),
                ("maxell", ctypes.c_int), ("precision", ctypes.c_int),
                ("want_rr", ctypes.c_int), ("data", CatalogSpec),
                ("randoms", CatalogSpec)]


class JobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int), ("status", ctypes.c_int),
                ("queued_s", ctypes.c_double), ("run_s", ctypes.c_double),
                ("latency_s", ctypes.c_double), ("footprint", ctypes.c_size_t),
                ("nrows", ctypes.c_int), ("nr", ctypes.c_int), ("nk", ctypes.c_int),
                ("has_rr", ctypes.c_int), ("data", AssignStats),
                ("randoms", AssignStats), ("phase_s", ctypes.c_double * 8),
                ("message", ctypes.c_char * 256)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_int), ("running", ctypes.c_int),
                ("peak_running", ctypes.c_int), ("resident_objects", ctypes.c_int),
                ("completed", ctypes.c_uint64),
                ("admitted_out_of_order", ctypes.c_uint64),
                ("evictions", ctypes.c_uint64), ("bytes_resident", ctypes.c_size_t),
                ("bytes_transient", ctypes.c_size_t), ("peak_bytes", ctypes.c_size_t),
                ("budget", ctypes.c_size_t)]


# name -> (restype, argtypes); every fc_* entry returns an fc_status int.
_SIGNATURES = {
    "fc_last_error": (ctypes.c_char_p, []),
    "fc_version": (ctypes.c_int, []),
    "fc_launch_count": (ctypes.c_int, [ctypes.POINTER(ctypes.c_ulonglong)]),
    "fc_profiler_range": (ctypes.c_int, [ctypes.c_int]),
    "fc_set_device": (ctypes.c_int, [ctypes.c_int]),
    "fc_grid_create": (ctypes.c_int, [c_int_p, c_double_p, ctypes.c_double, c_void_pp]),
    "fc_grid_create_precision": (ctypes.c_int, [c_int_p, c_double_p, ctypes.c_double,
                                                ctypes.c_int, c_void_pp]),
    "fc_grid_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "fc_grid_device_data": (ctypes.c_int, [ctypes.c_void_p, c_void_pp]),
    "fc_grid_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_grid_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_grid_upload": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_grid_download": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_grid_device_ptr": (ctypes.c_int, [ctypes.c_void_p, c_void_pp]),
    "fc_grid_coords": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int,
                                      c_double_p, c_int_p]),
    "fc_grid_sum": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p]),
    "fc_grid_add_scalar": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "fc_grid_multiply_by": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "fc_grid_axpy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "fc_assignor_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int64, c_void_pp]),
    "fc_assignor_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_assignor_add_posw": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int64]),
    "fc_assignor_add_pos_weights": (ctypes.c_int, [ctypes.c_void_p, c_double_p,
                                                   c_double_p, ctypes.c_int64]),
    "fc_assignor_add_pos_weight": (ctypes.c_int, [ctypes.c_void_p, c_double_p,
                                                  ctypes.c_double, ctypes.c_int64]),
    "fc_assignor_add_posw_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_int64]),
    "fc_assignor_add_random": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64,
                                              ctypes.c_double, c_double_p,
                                              ctypes.c_uint64, ctypes.c_int64]),
    "fc_assignor_flush": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_assignor_clear": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_assignor_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AssignStats)]),
    "fc_assignor_buffer_size": (ctypes.c_int, [ctypes.c_void_p,
                                               ctypes.POINTER(ctypes.c_int64)]),
    "fc_corr_create": (ctypes.c_int, [ctypes.c_int, c_int_p, ctypes.c_double, c_double_p,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_uint, ctypes.c_int, c_void_pp]),
    "fc_corr_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_corr_dims": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_int_p, c_int_p,
                                    c_int_p]),
    "fc_corr_set_grid2": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_corr_set_grid2_grid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fc_corr_set_grid2_fft": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_corr_autocorrelate": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_corr_autocorrelate_grid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fc_corr_cross_correlate": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_corr_cross_correlate_grid": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fc_corr_results": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_int_p, c_double_p,
                                       c_double_p, c_int_p, c_double_p, c_double_p]),
    "fc_corr_timings_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(CorrTimings)]),
    "fc_corr_footprint": (ctypes.c_int, [ctypes.c_int, c_int_p, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]),
    "fc_corr_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fc_corr_autocorrelate_grid_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fc_corr_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_corr_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fc_corr_set_term_shard": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_int]),
    "fc_corr_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(KernelTime),
                                       ctypes.c_int, c_int_p]),
    "fc_sum_sumsq_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_double_p,
                                           c_double_p]),
    "fc_device_synchronize": (ctypes.c_int, []),
    "fc_host_register": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    "fc_host_unregister": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_device_malloc": (ctypes.c_int, [ctypes.c_size_t, c_void_pp]),
    "fc_device_free": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_fault_inject": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64]),
    "fc_set_device_budget": (ctypes.c_int, [ctypes.c_size_t]),
    "fc_device_bytes": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t)]),
    "fc_memcpy_htod": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "fc_memcpy_dtoh": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "fc_device_memory": (ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_size_t)]),
    "fc_timer_create": (ctypes.c_int, [c_void_pp]),
    "fc_timer_start": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_timer_stop": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_timer_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_catalog_uniform": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_double_p,
                                          c_double_p, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_uint64]),
    "fc_catalog_clustered_box": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.c_double, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_uint64]),
    "fc_catalog_sector": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_uint64]),
    "fc_apply_displacement": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int64,
                                             c_double_p, ctypes.c_int, c_double_p]),
    "fc_catalog_generate": (ctypes.c_int, [ctypes.POINTER(CatalogSpec), ctypes.c_void_p]),
    "fc_job_init": (ctypes.c_int, [ctypes.POINTER(Job)]),
    "fc_job_footprint": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.POINTER(ctypes.c_size_t)]),
    "fc_server_create": (ctypes.c_int, [ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                        c_void_pp]),
    "fc_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Job),
                                        ctypes.POINTER(ctypes.c_uint64)]),
    "fc_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                      c_int_p]),
    "fc_server_job_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(JobInfo)]),
    "fc_server_job_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                             c_double_p, c_int_p, c_double_p, c_double_p,
                                             c_int_p, c_double_p, c_double_p]),
    "fc_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "fc_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "fc_batch_params_default": (ctypes.c_int, [ctypes.POINTER(BatchParams)]),
    "fc_batch_create": (ctypes.c_int, [ctypes.POINTER(BatchBox), ctypes.c_int,
                                       ctypes.POINTER(BatchParams), c_void_pp]),
    "fc_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_batch_run": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_batch_launch": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_batch_wait": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fc_batch_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchInfo)]),
    "fc_batch_box_dims": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_int_p,
                                         c_int_p]),
    "fc_batch_results": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p,
                                        c_int_p, c_double_p, c_double_p, c_int_p,
                                        c_double_p, c_double_p]),
    "fc_batch_box_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(AssignStats)]),
    "fc_tune_export": (ctypes.c_int, [ctypes.c_char_p]),
    "fc_tune_import": (ctypes.c_int, [ctypes.c_char_p]),
    "fc_tune_forget": (ctypes.c_int, []),
    "fc_tune_count": (ctypes.c_int, [c_int_p]),
    "fc_hist_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, c_void_pp]),
    "fc_hist_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_hist_nbins": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "fc_hist_accumulate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p,
                                          c_double_p, ctypes.c_int64]),
    "fc_hist_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "fc_hist_get": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_int_p, c_double_p]),
}

_lib = None


def load():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"fftcorr_b200 CUDA library missing at {LIB_PATH}; build it with "
            "`python -m fftcorr_b200._build` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    return list(_SIGNATURES)


def check(rc):
    """Raises the Python exception matching a non-zero fc_status."""
    if rc == FC_OK:
        return
    msg = load().fc_last_error().decode("utf-8", "replace")
    if rc == FC_ERR_INVALID:
        raise ValueError(msg)
    if rc == FC_ERR_RANGE:
        raise IndexError(msg)
    if rc == FC_ERR_ALLOC:
        raise MemoryError(msg)
    if rc == FC_ERR_ADMISSION:
        raise AdmissionError(rc, msg)
    raise FcError(rc, msg)


def call(name, *args):
    check(getattr(load(), name)(*args))


def launch_count():
    """This library's own kernel launches issued so far (see fc_api.h)."""
    n = ctypes.c_ulonglong()
    call("fc_launch_count", ctypes.byref(n))
    return n.value


def dptr(a):
    return a.ctypes.data_as(c_double_p)


def iptr(a):
    return a.ctypes.data_as(c_int_p)


def int3(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.intc).reshape(3))


def dbl3(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(3))
