"""B200 backend for RadiativeViewFactor.jl's element-pair view-factor assembly.

The package mirrors the reference's user-facing API for the GPU path
(compute_view_factors, register_gpu_hook, ViewFactorResult, check_reciprocity,
check_closure, aggregate_by_group; src/RadiativeViewFactor.jl:33-46) over the
C ABI of lib/librvf_b200.so (include/rvf_b200.h).  The directory name is not a
Python identifier; import it through importlib, e.g.

    spec = importlib.util.spec_from_file_location(
        "rvf_b200", "radiativeviewfactor.jl_b200/__init__.py",
        submodule_search_locations=["radiativeviewfactor.jl_b200"])
"""
from . import meshes, meshio
from ._abi import PinnedArray, RVFError, Session, DeviceMesh, load_library
from .assembly import (B200Backend, CPU, compute_view_factors, compute_view_factors_b200, make_options,
                       mesh_desc_arrays, register_gpu_hook)
from .mesh import FAMILY_CODES, MeshData, SurfaceElement, build_group_obs_soups, flatten, merged_obstruction
from .meshio import load_mesh, load_vtu
from .geometry import (element_area, line2_normal_and_length_element, line2_physical_point,
                       line3_normal_and_length_element, line3_physical_point, quad4_normal_and_area_element,
                       quad4_physical_point, quad8_normal_and_area_element, quad8_physical_point)
from .results import (ViewFactorResult, aggregate_by_group, check_closure, check_reciprocity,
                      reciprocity_error)

__all__ = [
    "B200Backend", "CPU", "DeviceMesh", "FAMILY_CODES", "MeshData", "PinnedArray", "RVFError", "Session",
    "SurfaceElement", "ViewFactorResult", "aggregate_by_group", "build_group_obs_soups", "check_closure",
    "check_reciprocity", "compute_view_factors", "compute_view_factors_b200", "element_area", "flatten",
    "line2_normal_and_length_element", "line2_physical_point", "line3_normal_and_length_element",
    "line3_physical_point", "load_library", "load_mesh", "load_vtu", "make_options", "merged_obstruction",
    "mesh_desc_arrays", "meshes", "meshio", "plot_mesh_normals", "quad4_normal_and_area_element",
    "quad4_physical_point", "quad8_normal_and_area_element", "quad8_physical_point", "reciprocity_error",
    "register_gpu_hook",
]


def plot_mesh_normals(mesh, *args, **kwargs):
    """src/RadiativeViewFactor.jl:48-56: the reference's Plots.jl extension
    (visualisation, not part of the assembly); not provided by this backend."""
    raise NotImplementedError("plot_mesh_normals is the reference's Plots.jl extension (visualisation); "
                              "this backend does not provide it.")
