"""spinfemx_b200: B200-native demag + LLG hot path of SpinFEMx behind a C ABI.

Lazy facade mirroring ``spinfemx.gpu`` (src/spinfemx/gpu/__init__.py:23-72): the
public names resolve on first access, so importing the package does not load
libspx.so or touch a GPU.
"""
from __future__ import annotations

import importlib

__version__ = "0.1.0"

_EXPORTS = {
    "DemagFieldLindholmGPU": ".demag",
    "EffectiveField": ".llg",
    "JvContext": ".llg",
    "EffectiveFieldSTTGPU": ".llg",
    "EffectiveFieldSOTGPU": ".llg",
    "JvContextSTT": ".llg",
    "JvContextSOT": ".llg",
    "LLG_GPU": ".llg",
    "HMatrixGPUPackedFused": ".hmatrix",
    "HMatrixBuildConfig": ".hmatrix",
    "build_or_load_hmatrix": ".hmatrix",
    "BoundaryGeometry": ".geometry",
    "kuhn_box": ".geometry",
    "boundary_data": ".geometry",
    "fem_assemble": ".geometry",
    "cluster_tree_perm": ".geometry",
    "dense_b_apply": ".geometry",
    "LLGEnsemble": ".ensemble",
    "EnergyMinimizerGPU": ".minimizer",
    "LaBonteBBMinimizerGPU": ".minimizer",
    "ensemble_mesh": ".ensemble",
    "read_xdmf_mesh": ".io",
    "read_hdf5": ".io",
    "XDMFWriter": ".io",
    "llg_trajectory": ".adjoint",
    "trajectory_tangent": ".adjoint",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name in _EXPORTS:
        mod = importlib.import_module(_EXPORTS[name], __name__)
        return getattr(mod, name)
    raise AttributeError(name)
