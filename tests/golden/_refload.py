"""Load individual beamz source files by path, under the numpy ``jax`` stand-in.

Fixture generation only (``make_golden.py``).  Package ``__init__`` files of
beamz import the whole framework (geometry, shapely, plotting), so they are
bypassed: empty package modules are registered for ``beamz``,
``beamz.simulation``, ``beamz.devices`` ... and each needed source file is
executed from the reference tree as its own module.  Names that a loaded file
imports from modules outside the step math are supplied as small stubs
(``model.CpmlPackedSlabSpec``/``CpmlTerm`` keep their reference field order).
"""

from __future__ import annotations

import importlib.util
import os
import sys
import types
from dataclasses import dataclass
from typing import Any, NamedTuple

from . import _jaxshim


def reference_root() -> str:
    """The beamz source tree: BEAMZ_REFERENCE_ROOT (the scripts set it from --reference)."""
    root = os.environ.get("BEAMZ_REFERENCE_ROOT")
    if not root:
        raise RuntimeError("set BEAMZ_REFERENCE_ROOT (or pass --reference) to the root of the beamz source tree")
    return root


def _package(name: str, path: str | None = None) -> types.ModuleType:
    mod = sys.modules.get(name)
    if mod is None:
        mod = types.ModuleType(name)
        mod.__path__ = [path] if path else []
        sys.modules[name] = mod
    return mod


def _load(name: str, relpath: str) -> types.ModuleType:
    if name in sys.modules and getattr(sys.modules[name], "__file__", None):
        return sys.modules[name]
    path = os.path.join(reference_root(), relpath)
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    sys.modules[name] = module
    spec.loader.exec_module(module)
    return module


class CpmlPackedSlabSpec(NamedTuple):
    """Field order of ``beamz/simulation/model.py:306-311``."""

    axis: int
    low: int
    high: int
    shape: tuple
    logical_stop: int = -1


@dataclass(frozen=True, eq=False)
class CpmlTerm:
    """Field order of ``beamz/simulation/model.py:314-324``."""

    component: str
    axis: int
    sign: float
    a: Any
    b: Any
    inv_kappa: Any
    slab: CpmlPackedSlabSpec


def load_reference():
    """Return a namespace with the reference modules the fixtures exercise."""
    _jaxshim.install()
    root = reference_root()
    _package("beamz", os.path.join(root, "beamz"))
    _package("beamz.simulation", os.path.join(root, "beamz/simulation"))
    _package("beamz.devices", os.path.join(root, "beamz/devices"))
    _package("beamz.devices.sources", os.path.join(root, "beamz/devices/sources"))
    _package("beamz.devices.monitors", os.path.join(root, "beamz/devices/monitors"))
    _package("beamz.design", os.path.join(root, "beamz/design"))

    const = _load("beamz.const", "beamz/const.py")
    lattice = _load("beamz.lattice", "beamz/lattice.py")

    model = types.ModuleType("beamz.simulation.model")
    model.CpmlPackedSlabSpec = CpmlPackedSlabSpec
    model.CpmlTerm = CpmlTerm
    for name in ("BoundaryPlan", "RunConfig", "SimulationState", "UpdateCoefficients"):
        setattr(model, name, type(name, (), {}))
    sys.modules["beamz.simulation.model"] = model

    kernels = _load("beamz.simulation.kernels", "beamz/simulation/kernels.py")

    immutable = _load("beamz.devices._immutable", "beamz/devices/_immutable.py")
    time_mod = _load("beamz.devices.sources.time", "beamz/devices/sources/time.py")

    discretization = types.ModuleType("beamz.design.discretization")
    discretization.MaterialGrid = type("MaterialGrid", (), {})
    sys.modules["beamz.design.discretization"] = discretization
    boundaries = _load("beamz.devices.boundaries", "beamz/devices/boundaries.py")
    boundary_compile = _load(
        "beamz.devices._boundary_compile", "beamz/devices/_boundary_compile.py"
    )

    # observe.py: only _accumulate_dft and its helpers are exercised; the other
    # names it imports belong to power/flux/recorder paths.
    mon_compiler = types.ModuleType("beamz.devices.monitors.compiler")
    mon_compiler.CompiledMonitorSpec = type("CompiledMonitorSpec", (), {})
    mon_compiler.__getattr__ = lambda name: type(name, (), {})
    sys.modules["beamz.devices.monitors.compiler"] = mon_compiler
    monitors = types.ModuleType("beamz.devices.monitors.monitors")
    monitors._line_integral_scale_2d = lambda *a, **k: None
    monitors._line_normal_2d = lambda *a, **k: None
    sys.modules["beamz.devices.monitors.monitors"] = monitors
    specs = types.ModuleType("beamz.devices.sources.specs")
    for name in ("GaussianBeamSource", "GaussianSource", "ModeSource"):
        setattr(specs, name, type(name, (), {}))
    sys.modules["beamz.devices.sources.specs"] = specs
    if not hasattr(lattice, "yee_flux"):
        lattice.yee_flux = lambda *a, **k: None
    model.SimulationState = type("SimulationState", (), {})
    observe = _load("beamz.simulation.observe", "beamz/simulation/observe.py")

    return types.SimpleNamespace(
        const=const,
        lattice=lattice,
        kernels=kernels,
        time=time_mod,
        boundaries=boundaries,
        boundary_compile=boundary_compile,
        observe=observe,
        immutable=immutable,
        jnp=sys.modules["jax.numpy"],
    )
