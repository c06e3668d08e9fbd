"""ctypes binding of liblbibcuda.so (the C ABI in include/lbibcell.h).

The shared library is built in-tree by lbibcell_b200/build.py.  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbibcuda.so")

#: symbols declared in include/lbibcell.h
SYMBOLS = (
    "lbib_create_from_files", "lbib_destroy", "lbib_step", "lbib_lattice_step", "lbib_get_sizes",
    "lbib_download_lattice", "lbib_upload_lattice", "lbib_download_membrane", "lbib_download_connections",
    "lbib_areas", "lbib_areas_static", "lbib_last_error", "lbib_last_timing", "lbib_set_profiling", "lbib_set_species_source",
    "lbib_get_domain_count", "lbib_diff_begin", "lbib_diff_forward", "lbib_diff_backward", "lbib_diff_end",
    "lbib_write_simulation", "lbib_load_solvers", "lbib_add_forces", "lbib_delete_force_type",
    "lbib_delete_all_forces", "lbib_nodes_within_radius", "lbib_closest_nodes", "lbib_write_vtk",
    "lbib_read_vtm_geometry", "lbib_upload_membrane", "lbib_cure_lattice", "lbib_accumulated_concentrations",
    "lbib_set_cell_types", "lbib_get_cell_types", "lbib_init_velocity", "lbib_diff_mass", "lbib_diff_fluid_seed",
    "lbib_diff_force_params", "lbib_diff_motion", "lbib_diff_positions", "lbib_download_forces", "lbib_set_species_sources",
)

_lib = None


class LbibError(RuntimeError):
    """An error code returned through the C ABI."""

    def __init__(self, code: int, message: str, index: int = -1):
        super().__init__(f"lbibcell error {code}: {message} (index {index})")
        self.code = code
        self.index = index


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lbibcell_b200.build` "
                          f"(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, cp = ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p
    L.lbib_create_from_files.restype = ip
    L.lbib_create_from_files.argtypes = [cp, cp, cp, cp, ip, ip, ctypes.POINTER(vp)]
    L.lbib_destroy.restype = ip
    L.lbib_destroy.argtypes = [vp]
    L.lbib_step.restype = ip
    L.lbib_step.argtypes = [vp, ip]
    L.lbib_lattice_step.restype = ip
    L.lbib_lattice_step.argtypes = [vp, ip, ip]
    L.lbib_get_sizes.restype = ip
    L.lbib_get_sizes.argtypes = [vp, vp]
    L.lbib_download_lattice.restype = ip
    L.lbib_download_lattice.argtypes = [vp] + [vp] * 6
    L.lbib_upload_lattice.restype = ip
    L.lbib_upload_lattice.argtypes = [vp, vp, vp, vp]
    L.lbib_init_velocity.restype = ip
    L.lbib_init_velocity.argtypes = [vp, ctypes.c_double, ctypes.c_double]
    L.lbib_download_membrane.restype = ip
    L.lbib_download_membrane.argtypes = [vp, vp, vp]
    L.lbib_download_connections.restype = ip
    L.lbib_download_connections.argtypes = [vp, vp]
    L.lbib_areas.restype = ip
    L.lbib_areas.argtypes = [vp, vp, vp, ip]
    L.lbib_areas_static.restype = ip
    L.lbib_areas_static.argtypes = [vp, vp, vp, ip]
    L.lbib_accumulated_concentrations.restype = ip
    L.lbib_accumulated_concentrations.argtypes = [vp, ctypes.c_char_p, vp, vp, ip]
    L.lbib_set_cell_types.restype = ip
    L.lbib_set_cell_types.argtypes = [vp, vp, vp, ip]
    L.lbib_get_cell_types.restype = ip
    L.lbib_get_cell_types.argtypes = [vp, vp, vp, ip]
    L.lbib_last_error.restype = ip
    L.lbib_last_error.argtypes = [vp, cp, ip, ctypes.POINTER(ctypes.c_longlong)]
    L.lbib_last_timing.restype = ip
    L.lbib_last_timing.argtypes = [vp, vp]
    L.lbib_set_species_source.restype = ip
    L.lbib_set_species_source.argtypes = [vp, ip, vp, ip]
    L.lbib_set_profiling.restype = ip
    L.lbib_set_profiling.argtypes = [vp, ip]
    L.lbib_get_domain_count.restype = ip
    L.lbib_get_domain_count.argtypes = [vp, ctypes.POINTER(ip)]
    L.lbib_diff_begin.restype = ip
    L.lbib_diff_begin.argtypes = [vp, ip, ip]
    L.lbib_diff_forward.restype = ip
    L.lbib_diff_forward.argtypes = [vp, vp, vp, vp, ip]
    L.lbib_diff_backward.restype = ip
    L.lbib_diff_backward.argtypes = [vp, vp, vp, vp, vp]
    L.lbib_diff_end.restype = ip
    L.lbib_diff_end.argtypes = [vp]
    L.lbib_diff_mass.restype = ip
    L.lbib_diff_mass.argtypes = [vp, vp, vp, ip]
    L.lbib_diff_fluid_seed.restype = ip
    L.lbib_diff_fluid_seed.argtypes = [vp, vp]
    L.lbib_set_species_sources.restype = ip
    L.lbib_set_species_sources.argtypes = [vp, vp, ip]
    L.lbib_diff_force_params.restype = ip
    L.lbib_diff_force_params.argtypes = [vp, vp, ip]
    L.lbib_diff_motion.restype = ip
    L.lbib_diff_motion.argtypes = [vp, ip, vp]
    L.lbib_diff_positions.restype = ip
    L.lbib_diff_positions.argtypes = [vp, vp, vp, ip]
    L.lbib_download_forces.restype = ip
    L.lbib_download_forces.argtypes = [vp, vp, vp, vp, vp, ip]
    L.lbib_write_simulation.restype = ip
    L.lbib_write_simulation.argtypes = [vp, cp, cp, cp, cp]
    L.lbib_load_solvers.restype = ip
    L.lbib_load_solvers.argtypes = [vp, cp]
    L.lbib_add_forces.restype = ip
    L.lbib_add_forces.argtypes = [vp, vp, vp, vp, vp, ip]
    L.lbib_delete_force_type.restype = ip
    L.lbib_delete_force_type.argtypes = [vp, ip]
    L.lbib_delete_all_forces.restype = ip
    L.lbib_delete_all_forces.argtypes = [vp]
    L.lbib_nodes_within_radius.restype = ip
    L.lbib_nodes_within_radius.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_longlong, vp, ip]
    L.lbib_cure_lattice.restype = ip
    L.lbib_cure_lattice.argtypes = [vp]
    L.lbib_upload_membrane.restype = ip
    L.lbib_upload_membrane.argtypes = [vp, vp, vp, ip, vp, ip]
    L.lbib_write_vtk.restype = ip
    L.lbib_write_vtk.argtypes = [vp, cp, ctypes.c_uint, ip, ip]
    L.lbib_read_vtm_geometry.restype = ip
    L.lbib_read_vtm_geometry.argtypes = [cp, vp, vp, ip, vp, ip, vp]
    L.lbib_closest_nodes.restype = ip
    L.lbib_closest_nodes.argtypes = [vp, vp, vp, vp, ip, ctypes.c_double, vp]
    _lib = L
    return L
