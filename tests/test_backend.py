"""Backend policy (beamz/simulation/backend.py:35-258 semantics): aliases,
environment defaults and flags, and resolution on a host without a B200
(auto falls back to beamz's JAX path; explicit requests raise)."""

from __future__ import annotations

import pytest

from beamz_b200 import abi
from beamz_b200 import backend as B


def test_aliases_and_environment_default(monkeypatch):
    assert B.normalize_backend("XLA") == "jax"
    for name in ("cuda", "streamed", "cuda_streamed", "cuda-streamed", "b200"):
        assert B.normalize_backend(name) == "b200"
    assert B.normalize_backend("hopper") == "cuda_hopper"
    monkeypatch.delenv("BEAMZ_EXECUTION_BACKEND", raising=False)
    assert B.normalize_backend(None) == "auto"
    monkeypatch.setenv("BEAMZ_EXECUTION_BACKEND", "jax")
    assert B.normalize_backend(None) == "jax"
    with pytest.raises(ValueError):
        B.normalize_backend("tpu")


def test_flags_from_environment(monkeypatch):
    monkeypatch.delenv("BEAMZ_CUDA_DISABLE_GRAPH_CACHE", raising=False)
    monkeypatch.delenv("BEAMZ_CUDA_CPML_PSI_PRECISION", raising=False)
    assert B.cuda_flags_from_env() == abi.FDTD_FLAG_GRAPH_CACHE
    monkeypatch.setenv("BEAMZ_CUDA_DISABLE_GRAPH_CACHE", "1")
    assert B.cuda_flags_from_env() == 0
    monkeypatch.setenv("BEAMZ_CUDA_DISABLE_GRAPH_CACHE", "off")
    assert B.cuda_flags_from_env() == abi.FDTD_FLAG_GRAPH_CACHE
    monkeypatch.setenv("BEAMZ_CUDA_CPML_PSI_PRECISION", "bf16")
    with pytest.raises(ValueError, match="FP32"):
        B.cuda_flags_from_env()
    monkeypatch.setenv("BEAMZ_CUDA_CPML_PSI_PRECISION", "fp16")
    with pytest.raises(ValueError):
        B.cuda_flags_from_env()


def test_resolution_without_a_b200(monkeypatch):
    status = B.BackendStatus(False, None, (), (), (), "no CUDA device is visible")
    monkeypatch.setattr(B, "backend_status", lambda: status)
    assert B.resolve_backend("jax") == "jax"
    assert B.resolve_backend("auto") == "jax"
    with pytest.raises(abi.CudaBackendUnavailable, match="no CUDA device"):
        B.resolve_backend("cuda")
    with pytest.raises(abi.CudaBackendUnavailable, match="sm_90"):
        B.resolve_backend("cuda_hopper")


def test_resolution_with_a_b200(monkeypatch):
    status = B.BackendStatus(True, abi.FDTD_ABI_VERSION, ("fdtd_phase", "fdtd_program"), ("NVIDIA B200",), (100,))
    monkeypatch.setattr(B, "backend_status", lambda: status)
    assert B.resolve_backend("auto") == "b200"
    assert B.resolve_backend("cuda_streamed") == "b200"
    assert B.resolve_backend("jax") == "jax"


def test_status_on_this_host_is_consistent():
    s = B.backend_status()
    if not s.available:
        assert s.reason
    else:
        assert s.compute_capabilities and all(c == 100 for c in s.compute_capabilities)
    assert set(s.as_dict()) == {"available", "abi_version", "targets", "gpu_devices", "compute_capabilities",
                                "reason"}


@pytest.mark.gpu
def test_the_engine_resolves_on_a_b200():
    s = B.backend_status()
    assert s.available, s.reason
    assert set(s.targets) == {"fdtd_phase", "fdtd_program"}
    assert B.resolve_backend("auto") == "b200"
