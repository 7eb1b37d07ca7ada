"""The C-ABI library: exports, struct layout and host-side validation (no GPU)."""

from __future__ import annotations

import ctypes
import os
import re

import pytest

from beamz_b200 import abi
from beamz_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdtd_b200.h")


@pytest.fixture(scope="module")
def lib():
    build()
    return abi.load_library()


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|void|const char\*|const FdtdRegistration\*)\s+(fdtd_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert names, "no declarations parsed"
    assert set(names) == set(abi.EXPORTED_SYMBOLS)
    for name in names:
        assert hasattr(lib, name), name


def test_registrations_table(lib):
    regs = abi.registrations(lib)
    assert set(regs) == {"fdtd_phase", "fdtd_program"}
    assert regs["fdtd_phase"] == ctypes.cast(lib.fdtd_launch_phase, ctypes.c_void_p).value
    assert regs["fdtd_program"] == ctypes.cast(lib.fdtd_launch_program, ctypes.c_void_p).value


def test_struct_layout_and_version(lib):
    assert lib.fdtd_abi_version() == abi.FDTD_ABI_VERSION
    assert lib.fdtd_program_size() == ctypes.sizeof(abi.FdtdProgram)


def _fake(shape, etype=abi.FDTD_F32, ptr=0x1000):
    b = abi.FdtdBuffer()
    b.data = ptr
    b.rank = len(shape)
    b.element_type = etype
    for i, n in enumerate(shape):
        b.dims[i] = n
    return b


def _valid_program():
    """A 3D voxel program with fake (never dereferenced) device pointers."""
    Z, Y, X = 4, 5, 6
    s = abi.FdtdProgram()
    s.abi_version = abi.FDTD_ABI_VERSION
    s.ndim = 3
    s.schedule = abi.FDTD_SCHEDULE_PHASES
    s.material_kind = abi.FDTD_MATERIAL_VOXEL
    s.cells[:] = [Z, Y, X]
    s.dt, s.resolution, s.inv_resolution = 1e-17, 2e-8, 5e7
    shapes = [(Z + 1, Y + 1, X), (Z + 1, Y, X + 1), (Z, Y + 1, X + 1), (Z, Y, X + 1), (Z, Y + 1, X), (Z + 1, Y, X)]
    for c, sh in enumerate(shapes):
        s.fields[c] = _fake(sh)
    for c in range(3):
        s.h_decay[c] = _fake(())
        s.h_source_site[c] = _fake(())
    s.voxels = _fake((Z, Y, X), abi.FDTD_U8)
    s.eps_table = _fake((256,))
    s.step_counter = _fake((1,), abi.FDTD_S32)
    s.step_time = _fake((8,))
    return s


def test_validate_accepts_a_consistent_program(lib):
    assert lib.fdtd_validate(ctypes.byref(_valid_program())) == 0


@pytest.mark.parametrize("mutate", [
    lambda s: setattr(s, "abi_version", 99),
    lambda s: setattr(s, "ndim", 4),
    lambda s: s.fields.__setitem__(1, _fake((5, 5, 6))),
    lambda s: s.fields.__setitem__(0, _fake((5, 6, 6), abi.FDTD_S32)),
    lambda s: setattr(s, "eps_table", _fake((255,))),
    lambda s: setattr(s, "voxels", _fake((4, 5, 6), abi.FDTD_F32)),
    lambda s: setattr(s, "schedule", abi.FDTD_SCHEDULE_FUSED),  # bank B missing
    lambda s: setattr(s, "source_count", 17),
    lambda s: setattr(s, "metallic_edges", 1 << 6),
    lambda s: setattr(s, "step_counter", _fake((1,), abi.FDTD_F32)),
])
def test_validate_rejects_inconsistent_programs(lib, mutate):
    s = _valid_program()
    mutate(s)
    assert lib.fdtd_validate(ctypes.byref(s)) == 1  # cudaErrorInvalidValue


def test_validate_checks_sources_and_cpml(lib):
    s = _valid_program()
    s.source_count = 1
    src = s.sources[0]
    src.component, src.timing = 1, abi.FDTD_TIMING_PRE_E
    src.start[:] = [4, 4, 6]
    src.coeff = _fake((1, 1, 1))
    src.waveform = _fake((3,))
    assert lib.fdtd_validate(ctypes.byref(s)) == 0
    src.start[:] = [4, 4, 7]  # past Ey's x extent (7)
    assert lib.fdtd_validate(ctypes.byref(s)) == 1
    src.start[:] = [0, 0, 0]
    src.timing = abi.FDTD_TIMING_H  # H timing on an E component
    assert lib.fdtd_validate(ctypes.byref(s)) == 1
    s = _valid_program()
    s.cpml = 1
    for t in range(6):
        s.h_terms[t].axis = (1, 0, 0, 2, 2, 1)[t]
        s.e_terms[t].axis = (1, 0, 0, 2, 2, 1)[t]
    assert lib.fdtd_validate(ctypes.byref(s)) == 0  # all slabs empty
    s.h_terms[0].low, s.h_terms[0].high = 1, 1
    assert lib.fdtd_validate(ctypes.byref(s)) == 1  # coefficient buffers missing
    for name in ("a", "b", "inv_kappa"):
        setattr(s.h_terms[0], name, _fake((2,)))
    s.h_terms[0].psi = _fake((4, 2, 7))  # Hx (4, 5, 7) with y -> 2
    assert lib.fdtd_validate(ctypes.byref(s)) == 0
    s.h_terms[0].axis = 2
    assert lib.fdtd_validate(ctypes.byref(s)) == 1


def test_runtime_refuses_cpu_devices():
    torch = pytest.importorskip("torch")
    from beamz_b200 import runtime
    from tests.scenarios import scenario_3d

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(abi.CudaBackendUnavailable):
        runtime.compile_program(scenario_3d(), device="cpu")


def _pitched_program():
    """A 3D fused program on the pitched layout with the site codebook."""
    Z, Y, X = 4, 5, 6
    pitch = 8
    s = _valid_program()
    s.schedule = abi.FDTD_SCHEDULE_FUSED
    s.layout = abi.FDTD_LAYOUT_PITCHED
    s.material_kind = abi.FDTD_MATERIAL_CODEBOOK
    s.pitch = pitch
    for c in range(6):
        s.fields[c] = _fake((Z + 1, Y + 1, pitch), ptr=0x1000 * (c + 1))
        s.fields_alt[c] = _fake((Z + 1, Y + 1, pitch), ptr=0x10000 * (c + 1))
    s.voxels = abi.FdtdBuffer()
    s.eps_table = abi.FdtdBuffer()
    s.site_ids = _fake((Z + 1, Y + 1, pitch), abi.FDTD_S32, ptr=0x200000)
    s.site_coef = _fake((3, 256))
    return s


def test_validate_pitched_codebook_program(lib):
    assert lib.fdtd_validate(ctypes.byref(_pitched_program())) == 0


@pytest.mark.parametrize("mutate", [
    lambda s: setattr(s, "pitch", 6),                                     # < X + 1
    lambda s: setattr(s, "pitch", 9),                                     # not a multiple of 4
    lambda s: setattr(s, "site_ids", _fake((5, 6, 8), abi.FDTD_F32)),     # wrong type
    lambda s: setattr(s, "site_ids", _fake((5, 6, 8), abi.FDTD_S32, ptr=0x1004)),  # misaligned
    lambda s: setattr(s, "site_coef", _fake((256,))),
    lambda s: setattr(s, "material_kind", abi.FDTD_MATERIAL_VOXEL),       # pitched needs the codebook
    lambda s: setattr(s, "layout", abi.FDTD_LAYOUT_DENSE),                # codebook needs pitched
    lambda s: s.h_decay.__setitem__(0, _fake((4, 5, 7))),                 # non-uniform H
])
def test_validate_rejects_inconsistent_pitched_programs(lib, mutate):
    s = _pitched_program()
    mutate(s)
    assert lib.fdtd_validate(ctypes.byref(s)) == 1
