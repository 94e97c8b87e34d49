"""bismit_b200: bismit's per-area cortical cycle plus learning on NVIDIA B200.

The hot path (synapse gather, dendrite and tuft reductions, hex inhibition,
spiny-stellate and pyramidal learning) is hand-written sm_100a CUDA in
libbismit_b200.so behind the C ABI of include/bismit_b200.h. This package is
the host side above that ABI: the scheme builders of bismit's `map` module and
the Cortex / CorticalArea objects. There is no CPU fallback: using a Cortex
without the built library raises ImportError.
"""
from . import _ffi
from ._ffi import BismitError
from .cortex import Cortex, CortexBuilder, CorticalArea
from .map import (AreaScheme, AreaSchemeList, AxonDomain, AxonTopology, CellScheme, ControlCellKind,
                  CorticalAreaSettings, InputTrack, LayerMapKind, LayerMapScheme, LayerMapSchemeList,
                  LayerScheme, LayerTags, THAL_NSP, THAL_SP, TuftScheme, TuftSourceLayer, area_desc)

__all__ = [
    "AreaScheme", "AreaSchemeList", "AxonDomain", "AxonTopology", "BismitError", "CellScheme",
    "ControlCellKind", "Cortex", "CortexBuilder", "CorticalArea", "CorticalAreaSettings", "InputTrack",
    "LayerMapKind", "LayerMapScheme", "LayerMapSchemeList", "LayerScheme", "LayerTags", "THAL_NSP",
    "THAL_SP", "TuftScheme", "TuftSourceLayer", "area_desc",
]


def plan_of(desc, seed=0):
    """Resolves a bm_area_desc into its bm_area_plan without touching a device."""
    import ctypes as C
    p = _ffi.bm_area_plan()
    _ffi.check(_ffi.lib().bm_plan_resolve(C.byref(desc), C.c_uint64(seed), C.byref(p)))
    return p
