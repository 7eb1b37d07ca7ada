"""ctypes mirror of ``include/fdtd_b200.h`` and the library loader.

The library is built in-tree (``beamz_b200/_fdtd_b200.so``).  Loading checks
the ABI version and ``sizeof(FdtdProgram)`` against this mirror before any
launch, the way beamz validates its extension manifest
(beamz/simulation/backend.py:139-157).  There is no fallback: when the library
is missing or mismatched, :class:`CudaBackendUnavailable` is raised.
"""

from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_fdtd_b200.so")

FDTD_ABI_VERSION = 13
FDTD_F32, FDTD_S32, FDTD_BF16, FDTD_U8, FDTD_F64 = 0, 1, 2, 3, 4
FDTD_FLAG_GRAPH_CACHE = 1 << 7
FDTD_FLAG_DFT_OVERLAP = 1 << 16
FDTD_FLAG_CLASSES = 1 << 17
FDTD_FLAG_FAST_MATH = 1 << 19
FDTD_FLAG_LOSSY = 1 << 20
FDTD_FLAG_TEST_STALL = 1 << 18
FDTD_SCHEDULE_PHASES, FDTD_SCHEDULE_FUSED = 0, 1
FDTD_MATERIAL_SITE, FDTD_MATERIAL_VOXEL, FDTD_MATERIAL_CODEBOOK = 0, 1, 2
FDTD_LAYOUT_DENSE, FDTD_LAYOUT_PITCHED = 0, 1
FDTD_TIMING_PRE_E, FDTD_TIMING_H, FDTD_TIMING_E = 0, 1, 2
FDTD_MAX_SOURCES = 16
FDTD_MAX_MONITORS = 16
FDTD_ADJOINT_NOALLOC_MAX_FLOATS = 4 * 1024 * 1024
FDTD_DIAG_BLOCKS = 592
TIMINGS = {"pre_e": FDTD_TIMING_PRE_E, "h": FDTD_TIMING_H, "e": FDTD_TIMING_E}
# Wall bits (front, back, bottom, top, left, right), beamz/simulation/cuda/runtime.py:38-40.
EDGE_BITS = {"front": 0, "back": 1, "bottom": 2, "top": 3, "left": 4, "right": 5}

#: Every symbol ``include/fdtd_b200.h`` declares.
EXPORTED_SYMBOLS = (
    "fdtd_abi_version",
    "fdtd_program_size",
    "fdtd_validate",
    "fdtd_launch_phase",
    "fdtd_launch_program",
    "fdtd_apply_sources",
    "fdtd_accumulate_dft",
    "fdtd_record_fields",
    "fdtd_copy_component",
    "fdtd_adjoint_step",
    "fdtd_adjoint_curl",
    "fdtd_field_diagnostics",
    "fdtd_dft_change",
    "fdtd_pack_gather",
    "fdtd_voxel_histogram",
    "fdtd_monitor_reduce",
    "fdtd_adjoint_step_noalloc",
    "fdtd_graph_create",
    "fdtd_graph_launch",
    "fdtd_graph_destroy",
    "fdtd_clear_graph_cache",
    "fdtd_error_string",
    "fdtd_registrations",
)


class CudaBackendUnavailable(RuntimeError):
    """The native library is missing, mismatched, or no CUDA device is usable."""


class FdtdError(RuntimeError):
    """A native call returned a non-zero CUDA error code."""

    def __init__(self, code: int, name: str, where: str):
        super().__init__(f"{where} failed: {code} ({name})")
        self.code = code
        self.name = name


class FdtdBuffer(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("rank", ctypes.c_int32),
        ("element_type", ctypes.c_int32),
        ("dims", ctypes.c_int64 * 4),
    ]


class FdtdCpmlTerm(ctypes.Structure):
    _fields_ = [
        ("axis", ctypes.c_int32),
        ("low", ctypes.c_int32),
        ("high", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("a", FdtdBuffer),
        ("b", FdtdBuffer),
        ("inv_kappa", FdtdBuffer),
        ("psi", FdtdBuffer),
        ("psi_alt", FdtdBuffer),
    ]


class FdtdSource(ctypes.Structure):
    _fields_ = [
        ("component", ctypes.c_int32),
        ("timing", ctypes.c_int32),
        ("start", ctypes.c_int32 * 3),
        ("reserved", ctypes.c_int32),
        ("coeff", FdtdBuffer),
        ("waveform", FdtdBuffer),
    ]


class FdtdDft(ctypes.Structure):
    _fields_ = [
        ("monitor_count", ctypes.c_int32),
        ("batch", ctypes.c_int32),
        ("indices", FdtdBuffer),
        ("weights", FdtdBuffer),
        ("freqs", FdtdBuffer),
        ("masks", FdtdBuffer),
        ("counts", FdtdBuffer),
        ("codes", FdtdBuffer),
        ("windows", FdtdBuffer),
        ("re", FdtdBuffer),
        ("im", FdtdBuffer),
        ("weight_sum", FdtdBuffer),
        ("samples", FdtdBuffer),
        ("affine", FdtdBuffer),
    ]


class FdtdAdjointStep(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("step", ctypes.c_int32),
        ("scratch_e", FdtdBuffer * 6),
        ("scratch_h", FdtdBuffer * 6),
        ("dft_grad_re", FdtdBuffer),
        ("dft_grad_im", FdtdBuffer),
        ("curl", FdtdBuffer * 3),
        ("grad", FdtdBuffer * 3),
        ("box_lo", ctypes.c_int32 * 3),
        ("box_hi", ctypes.c_int32 * 3),
    ]


class FdtdDiagnostics(ctypes.Structure):
    _fields_ = [
        ("site_eps_table", FdtdBuffer),
        ("site_eps", FdtdBuffer * 3),
        ("partials", FdtdBuffer),
        ("out", FdtdBuffer),
    ]


class FdtdDftChange(ctypes.Structure):
    _fields_ = [("prev_re", FdtdBuffer), ("prev_im", FdtdBuffer), ("out", FdtdBuffer)]


class FdtdGatherPack(ctypes.Structure):
    _fields_ = [
        ("indices_in", FdtdBuffer),
        ("weights_in", FdtdBuffer),
        ("indices_out", FdtdBuffer),
        ("weights_out", FdtdBuffer),
        ("dims", ctypes.c_int32 * 3),
        ("row", ctypes.c_int64),
        ("plane", ctypes.c_int64),
    ]


class FdtdMonitorReduce(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("freq_count", ctypes.c_int32),
        ("value_offset", ctypes.c_int64),
        ("point_count", ctypes.c_int64),
        ("e", ctypes.c_int32 * 2),
        ("h", ctypes.c_int32 * 2),
        ("rows", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("scale", FdtdBuffer),
        ("weights", FdtdBuffer),
        ("profile_re", FdtdBuffer),
        ("profile_im", FdtdBuffer),
        ("out", FdtdBuffer),
    ]


class FdtdRegistration(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("fn", ctypes.c_void_p)]


FDTD_MAX_RECORDERS = 4


class FdtdRecorder(ctypes.Structure):
    _fields_ = [
        ("interval", ctypes.c_int32),
        ("capacity", ctypes.c_int32),
        ("component_count", ctypes.c_int32),
        ("components", ctypes.c_int32 * 6),
        ("signs", ctypes.c_float * 6),
        ("indices", FdtdBuffer * 6),
        ("weights", FdtdBuffer * 6),
        ("values", FdtdBuffer * 6),
        ("steps", FdtdBuffer),
        ("times", FdtdBuffer),
        ("count", FdtdBuffer),
    ]


class FdtdProgram(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("ndim", ctypes.c_int32),
        ("polarization", ctypes.c_int32),
        ("schedule", ctypes.c_int32),
        ("material_kind", ctypes.c_int32),
        ("metallic_edges", ctypes.c_int32),
        ("cpml", ctypes.c_int32),
        ("nsteps", ctypes.c_int32),
        ("source_count", ctypes.c_int32),
        ("cells", ctypes.c_int64 * 3),
        ("dt", ctypes.c_float),
        ("resolution", ctypes.c_float),
        ("inv_resolution", ctypes.c_float),
        ("dt_over_eps", ctypes.c_float),
        ("dt_over_mu", ctypes.c_float),
        ("h_source", ctypes.c_float),
        ("tile_x", ctypes.c_int32),
        ("tile_y", ctypes.c_int32),
        ("z_chunk", ctypes.c_int32),
        ("layout", ctypes.c_int32),
        ("pitch", ctypes.c_int64),
        ("wait_limit_ns", ctypes.c_int64),
        ("fields", FdtdBuffer * 6),
        ("fields_alt", FdtdBuffer * 6),
        ("e_decay", FdtdBuffer * 3),
        ("e_source", FdtdBuffer * 3),
        ("h_decay", FdtdBuffer * 3),
        ("h_source_site", FdtdBuffer * 3),
        ("voxels", FdtdBuffer),
        ("eps_table", FdtdBuffer),
        ("site_ids", FdtdBuffer),
        ("site_coef", FdtdBuffer),
        ("h_terms", FdtdCpmlTerm * 6),
        ("e_terms", FdtdCpmlTerm * 6),
        ("sources", FdtdSource * FDTD_MAX_SOURCES),
        ("dft", FdtdDft),
        ("step_counter", FdtdBuffer),
        ("step_time", FdtdBuffer),
        ("status", FdtdBuffer),
        ("metric_h", FdtdBuffer * 3),
        ("metric_e", FdtdBuffer * 3),
        ("recorder_count", ctypes.c_int32),
        ("reserved_recorders", ctypes.c_int32),
        ("recorders", FdtdRecorder * FDTD_MAX_RECORDERS),
        ("site_class", FdtdBuffer),
        ("class_coef", FdtdBuffer),
        ("h_class", FdtdBuffer),
        ("h_class_coef", FdtdBuffer),
    ]


_TORCH_DTYPES = None


def buffer_of(tensor) -> FdtdBuffer:
    """Describe a contiguous torch tensor (device memory) as an FdtdBuffer."""
    global _TORCH_DTYPES
    import torch

    if _TORCH_DTYPES is None:
        _TORCH_DTYPES = {torch.float32: FDTD_F32, torch.int32: FDTD_S32, torch.bfloat16: FDTD_BF16,
                         torch.uint8: FDTD_U8, torch.float64: FDTD_F64}
    buf = FdtdBuffer()
    if tensor is None:
        return buf
    if not tensor.is_contiguous():
        raise ValueError("FDTD buffers must be contiguous")
    if tensor.dim() > 4:
        raise ValueError("FDTD buffers have rank <= 4")
    buf.data = tensor.data_ptr() if tensor.numel() else None
    buf.rank = tensor.dim()
    buf.element_type = _TORCH_DTYPES[tensor.dtype]
    for a, n in enumerate(tensor.shape):
        buf.dims[a] = int(n)
    return buf


_LIB = None
_LOCK = threading.Lock()


def load_library(path: str | None = None):
    """Load and check the native library (no GPU needed)."""
    global _LIB
    with _LOCK:
        if _LIB is not None and path is None:
            return _LIB
        lib_path = path or LIB_PATH
        if not os.path.exists(lib_path):
            raise CudaBackendUnavailable(
                f"{lib_path} is missing; build it with `python -m beamz_b200.build`"
            )
        try:
            lib = ctypes.CDLL(lib_path)
        except OSError as exc:  # pragma: no cover - loader failure
            raise CudaBackendUnavailable(f"cannot load {lib_path}: {exc}") from exc
        for name in EXPORTED_SYMBOLS:
            if not hasattr(lib, name):
                raise CudaBackendUnavailable(f"{lib_path} does not export {name}")
        lib.fdtd_abi_version.restype = ctypes.c_int
        lib.fdtd_program_size.restype = ctypes.c_int64
        lib.fdtd_validate.argtypes = [ctypes.POINTER(FdtdProgram)]
        lib.fdtd_validate.restype = ctypes.c_int
        lib.fdtd_launch_phase.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.c_int32]
        lib.fdtd_launch_phase.restype = ctypes.c_int
        lib.fdtd_launch_program.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram)]
        lib.fdtd_launch_program.restype = ctypes.c_int
        lib.fdtd_apply_sources.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.c_int32,
                                           ctypes.c_int32]
        lib.fdtd_apply_sources.restype = ctypes.c_int
        lib.fdtd_accumulate_dft.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.c_int32]
        lib.fdtd_accumulate_dft.restype = ctypes.c_int
        lib.fdtd_record_fields.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.c_int32]
        lib.fdtd_record_fields.restype = ctypes.c_int
        lib.fdtd_copy_component.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdBuffer), ctypes.POINTER(FdtdBuffer),
                                            ctypes.POINTER(ctypes.c_int64)]
        lib.fdtd_copy_component.restype = ctypes.c_int
        lib.fdtd_adjoint_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.POINTER(FdtdAdjointStep)]
        lib.fdtd_adjoint_step.restype = ctypes.c_int
        lib.fdtd_adjoint_curl.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.POINTER(FdtdAdjointStep)]
        lib.fdtd_adjoint_curl.restype = ctypes.c_int
        lib.fdtd_adjoint_step_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram),
                                                  ctypes.POINTER(FdtdAdjointStep)]
        lib.fdtd_adjoint_step_noalloc.restype = ctypes.c_int
        lib.fdtd_field_diagnostics.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram),
                                               ctypes.POINTER(FdtdDiagnostics)]
        lib.fdtd_field_diagnostics.restype = ctypes.c_int
        lib.fdtd_dft_change.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.POINTER(FdtdDftChange)]
        lib.fdtd_dft_change.restype = ctypes.c_int
        lib.fdtd_pack_gather.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdGatherPack)]
        lib.fdtd_pack_gather.restype = ctypes.c_int
        lib.fdtd_voxel_histogram.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdBuffer), ctypes.POINTER(FdtdBuffer)]
        lib.fdtd_voxel_histogram.restype = ctypes.c_int
        lib.fdtd_monitor_reduce.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram),
                                            ctypes.POINTER(FdtdMonitorReduce)]
        lib.fdtd_monitor_reduce.restype = ctypes.c_int
        lib.fdtd_graph_create.argtypes = [ctypes.c_void_p, ctypes.POINTER(FdtdProgram), ctypes.POINTER(ctypes.c_void_p)]
        lib.fdtd_graph_create.restype = ctypes.c_int
        lib.fdtd_graph_launch.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.fdtd_graph_launch.restype = ctypes.c_int
        lib.fdtd_graph_destroy.argtypes = [ctypes.c_void_p]
        lib.fdtd_graph_destroy.restype = ctypes.c_int
        lib.fdtd_clear_graph_cache.restype = None
        lib.fdtd_error_string.argtypes = [ctypes.c_int]
        lib.fdtd_error_string.restype = ctypes.c_char_p
        lib.fdtd_registrations.argtypes = [ctypes.POINTER(ctypes.c_int32)]
        lib.fdtd_registrations.restype = ctypes.POINTER(FdtdRegistration)
        version = lib.fdtd_abi_version()
        if version != FDTD_ABI_VERSION:
            raise CudaBackendUnavailable(f"ABI mismatch: library {version}, bindings {FDTD_ABI_VERSION}")
        size = lib.fdtd_program_size()
        if size != ctypes.sizeof(FdtdProgram):
            raise CudaBackendUnavailable(
                f"FdtdProgram layout mismatch: library {size} bytes, bindings {ctypes.sizeof(FdtdProgram)}"
            )
        if path is None:
            _LIB = lib
        return lib


def registrations(lib=None) -> dict:
    """Target name -> entry-point address, from the library's own table."""
    lib = lib or load_library()
    n = ctypes.c_int32(0)
    table = lib.fdtd_registrations(ctypes.byref(n))
    return {table[i].name.decode(): table[i].fn for i in range(n.value)}


def check(code: int, where: str) -> None:
    if code != 0:
        lib = load_library()
        name = lib.fdtd_error_string(int(code))
        raise FdtdError(int(code), name.decode() if name else "unknown", where)
