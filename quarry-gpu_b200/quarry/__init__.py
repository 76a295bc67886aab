"""quarry on B200: GPU spatial queries (LBVH / SAH build, rays, closest / kNN / radius).

The compiled module `_quarry` (csrc/quarry_py.cpp, over libquarry_b200.so) provides the
reference module's API: describe, demo_mesh, demo_gaussians, Scene, PointCloud and
GaussianCloud.  `quarry.capi` is the ctypes binding of the C ABI, `quarry.workloads` the
seeded benchmark inputs and `quarry.torch` the differentiable queries.
"""
from __future__ import annotations

try:
    from ._quarry import (  # noqa: F401
        GaussianCloud,
        PointCloud,
        Scene,
        __version__,
        demo_gaussians,
        demo_mesh,
        describe,
    )
    from . import zerocopy as _zerocopy

    _zerocopy.install(Scene, PointCloud, GaussianCloud)
except ImportError as _e:  # the extension is built by quarry-gpu_b200/build.py
    _import_error = _e

    _API = {"GaussianCloud", "PointCloud", "Scene", "__version__", "demo_gaussians",
            "demo_mesh", "describe"}

    def __getattr__(name):
        if name in _API:
            raise ImportError(f"quarry extension not built ({_import_error}); "
                              "run python quarry-gpu_b200/build.py")
        raise AttributeError(name)
