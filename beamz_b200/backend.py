"""Backend policy for the engine, shaped like beamz's
(beamz/simulation/backend.py:35-258): which execution backend a request
resolves to, the environment's cache/precision flags, and a diagnostic status.

The engine stands in for beamz's streamed CUDA target: the names ``cuda``,
``cuda_streamed`` and ``streamed`` (and ``b200``) resolve to it.  ``auto``
takes it when the library loads and every visible GPU is a B200 (sm_100),
and otherwise leaves the simulation on beamz's own JAX path; an explicit
request that cannot run raises ``CudaBackendUnavailable``, never a silent
downgrade.  The Hopper target (``cuda_hopper``) belongs to beamz's sm_90
kernels and is not provided.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

from . import abi
from .abi import CudaBackendUnavailable

# beamz/simulation/backend.py:84-108, with this engine in the CUDA slots.
_ALIASES = {
    "auto": "auto",
    "jax": "jax",
    "xla": "jax",
    "cuda": "b200",
    "streamed": "b200",
    "cuda_streamed": "b200",
    "cuda-streamed": "b200",
    "b200": "b200",
    "hopper": "cuda_hopper",
    "cuda_hopper": "cuda_hopper",
    "cuda-hopper": "cuda_hopper",
}


def normalize_backend(backend: str | None) -> str:
    """The canonical backend name; None reads BEAMZ_EXECUTION_BACKEND (default auto)."""
    value = os.environ.get("BEAMZ_EXECUTION_BACKEND", "auto") if backend is None else str(backend)
    try:
        return _ALIASES[value.strip().lower()]
    except KeyError as exc:
        raise ValueError(f"Unknown execution backend {value!r}; use one of: auto, jax, cuda, cuda_streamed, "
                         "b200.") from exc


def _env_enabled(name: str, default: bool) -> bool:
    value = os.environ.get(name)
    if value is None or not value.strip():
        return default
    return value.strip().lower() not in {"0", "false", "no", "off"}


def cuda_flags_from_env() -> int:
    """FdtdProgram.flags from the environment (beamz/simulation/backend.py:46-56):
    the graph cache unless BEAMZ_CUDA_DISABLE_GRAPH_CACHE is set.  ψ stays
    FP32: BEAMZ_CUDA_CPML_PSI_PRECISION=bf16 is refused (no BF16 storage)."""
    flags = abi.FDTD_FLAG_GRAPH_CACHE
    if _env_enabled("BEAMZ_CUDA_DISABLE_GRAPH_CACHE", False):
        flags &= ~abi.FDTD_FLAG_GRAPH_CACHE
    precision = os.environ.get("BEAMZ_CUDA_CPML_PSI_PRECISION", "fp32").strip().lower()
    if precision in {"bf16", "bfloat16"}:
        raise ValueError("beamz_b200 keeps CPML psi in FP32; BF16 psi storage is not provided")
    if precision not in {"fp32", "float32", ""}:
        raise ValueError("BEAMZ_CUDA_CPML_PSI_PRECISION must be 'fp32' or 'bf16'")
    return flags


@dataclass(frozen=True)
class BackendStatus:
    """Diagnostic snapshot (beamz: CudaBackendStatus, backend.py:59-81)."""

    available: bool
    abi_version: int | None
    targets: tuple
    gpu_devices: tuple
    compute_capabilities: tuple
    reason: str | None = None

    def as_dict(self) -> dict:
        return {"available": self.available, "abi_version": self.abi_version, "targets": self.targets,
                "gpu_devices": self.gpu_devices, "compute_capabilities": self.compute_capabilities,
                "reason": self.reason}


def backend_status() -> BackendStatus:
    """Whether the engine can run here: the library loads with a matching ABI
    and struct size, and every visible GPU is sm_100 (the kernels are built
    for sm_100a only)."""
    try:
        import torch
    except ImportError as exc:  # pragma: no cover - torch is a dependency
        return BackendStatus(False, None, (), (), (), f"torch is unavailable: {exc}")
    names, caps = (), ()
    if torch.cuda.is_available():
        n = torch.cuda.device_count()
        names = tuple(torch.cuda.get_device_name(i) for i in range(n))
        caps = tuple(10 * a + b for a, b in (torch.cuda.get_device_capability(i) for i in range(n)))
    try:
        lib = abi.load_library()
        targets = tuple(sorted(abi.registrations(lib)))
    except (OSError, CudaBackendUnavailable, abi.FdtdError) as exc:
        return BackendStatus(False, None, (), names, caps, f"the beamz_b200 library is unavailable: {exc}")
    if not caps:
        return BackendStatus(False, abi.FDTD_ABI_VERSION, targets, names, caps, "no CUDA device is visible")
    if any(c != 100 for c in caps):
        return BackendStatus(False, abi.FDTD_ABI_VERSION, targets, names, caps,
                             "beamz_b200 kernels are built for sm_100a (B200) only")
    return BackendStatus(True, abi.FDTD_ABI_VERSION, targets, names, caps)


def resolve_backend(backend: str | None) -> str:
    """"jax" (beamz's own path) or "b200", without weakening an explicit
    request (beamz/simulation/backend.py:223-258)."""
    requested = normalize_backend(backend)
    if requested == "jax":
        return "jax"
    if requested == "cuda_hopper":
        raise CudaBackendUnavailable("cuda_hopper is beamz's sm_90 target; beamz_b200 provides the sm_100a "
                                     "engine as backend 'cuda' / 'b200'")
    status = backend_status()
    if status.available:
        return "b200"
    if requested == "auto":
        return "jax"
    raise CudaBackendUnavailable(f"the b200 execution backend was requested but is unavailable: {status.reason}. "
                                 "Build it with `python -m beamz_b200.build`, or use backend='jax'.")
