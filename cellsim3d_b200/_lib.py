"""ctypes binding of libcs3d.so (include/cs3d.h).  No fallback: importing
the functions below raises if the in-tree library is missing."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcs3d.so")

SLOTS = 192
NODES = 180

OK = 0
E_ARG, E_CUDA, E_NOMEM, E_IO, E_PARSE, E_CONFIG, E_DEVICE_FLAGS, E_UNSUPPORTED = -1, -2, -3, -4, -5, -6, -7, -8
E_CAPACITY = -69

ERRBITS = {0x001: "NAN", 0x002: "CAPACITY", 0x004: "CAND_OVERFLOW", 0x008: "ENTRY_OVERFLOW",
           0x010: "NONFINITE_VOL", 0x020: "BAD_NORMAL", 0x040: "GRID_OVERFLOW", 0x080: "PAIR_OVERFLOW",
           0x100: "HALO_OVERFLOW", 0x200: "SOFT_CELLS"}

OPT_RECORD_PAIRS, OPT_SKIN, OPT_PAIR_CAPACITY, OPT_REBUILD, OPT_HALO_STATS = 1, 2, 3, 4, 5


class Params(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "particle_mass", "repulsion_range", "attraction_range", "repulsion_strength",
        "attraction_strength", "youngs_mod", "stiffness1", "internal_damping", "viscotic_damping",
        "gamma_visc", "division_vol", "time_interval", "max_pressure", "min_pressure",
        "growth_rate", "thresh_dist")] + [("box_len", C.c_float * 3)] + [(n, C.c_int32) for n in (
        "check_sphericity", "constrain_angles", "use_rigid_box", "daught_same_stiffness",
        "div_time_steps", "rng_ij", "rng_kl", "add_rands")] + [("rand_scale_factor", C.c_float),
                                                             ("rand_seed", C.c_int32), ("correct_com", C.c_int32),
        ("use_different_stiffnesses", C.c_int32), ("stiffness2", C.c_float), ("phase_count", C.c_int32),
        ("soften_after_growth", C.c_int32), ("number_of_softer_cells", C.c_int32),
        ("fraction_of_softer_cells", C.c_float), ("choose_random_cell_indices", C.c_int32),
        ("closeness_to_center", C.c_float), ("count_internal_radius", C.c_float)]


class Topology(C.Structure):
    _fields_ = [("nn", C.c_int32 * 576), ("sign", C.c_int32 * 180), ("r0", C.c_float * 576),
                ("theta0", C.c_float * 576), ("faces", C.c_int32 * 644)]


class Mesh(C.Structure):
    _fields_ = [("xyz", C.c_float * 540), ("nn", C.c_int32 * 576), ("sign", C.c_int32 * 180),
                ("bonds", C.c_int32 * 540), ("faces", C.c_int32 * 644)]


class Rng(C.Structure):
    _fields_ = [("u", C.c_float * 98), ("c", C.c_float), ("cd", C.c_float), ("cm", C.c_float),
                ("i97", C.c_int32), ("j97", C.c_int32), ("ok", C.c_int32)]


_i, _f = C.c_int32, C.c_float
Config = type("Config", (C.Structure,), {"_fields_": [
    ("max_cells", _i), ("particle_mass", _f), ("repulsion_range", _f), ("attraction_range", _f),
    ("repulsion_strength", _f), ("attraction_strength", _f), ("youngs_mod", _f), ("stiff_factor1", _f),
    ("viscotic_damping", _f), ("internal_damping", _f), ("gamma_visc", _f), ("division_vol", _f),
    ("random_z_offset", _i), ("z_offset", _f), ("div_time_steps", _i), ("time_interval", _f),
    ("restart", _i), ("traj_write_int", _i), ("non_div_time_steps", _i),
    ("traj_file_name", C.c_char * 256), ("binary_output", _i),
    ("max_pressure", _f), ("min_pressure", _f), ("growth_rate", _f),
    ("check_sphericity", _i), ("constrain_angles", _i), ("do_adaptive_dt", _i),
    ("dt_max", _f), ("dt_tol", _f), ("phase_count", _i), ("write_cont_force", _i),
    ("forces_file", C.c_char * 256), ("correct_com", _i),
    ("mit_index_file", C.c_char * 256), ("count_only_internal", _i), ("radius_cutoff", _f),
    ("overwrite_mit_ind", _i), ("cell_count_int", _i),
    ("do_pop_model", _i), ("total_food", _f), ("regular_consumption", _f), ("division_consumption", _f),
    ("death_release_food", _f), ("cell_life_time", _i), ("max_pop", _f),
    ("use_walls", _i), ("perp_axis", C.c_char * 8), ("d_axis", _f), ("wall_len", _f), ("wall_width", _f),
    ("thresh_dist", _f),
    ("use_div_plane_basis", _i), ("div_plane_basis", _f * 3),
    ("use_different_stiffnesses", _i), ("soft_stiff_factor", _f), ("number_of_softer_cells", _i),
    ("fraction_of_softer_cells", _f), ("during_growth", _i), ("daught_same_stiffness", _i),
    ("closeness_to_center", _f), ("start_at_pop", _i), ("choose_random_cell_indices", _i), ("recalc_r0", _i),
    ("use_rigid_box", _i), ("use_pbcs", _i), ("box_length", _f), ("box_len", _f * 3),
    ("flatbox", _i), ("rand_pos", _i),
    ("add_rands", _i), ("rand_seed", _i), ("rand_dist", _i), ("rand_scale_factor", _f)]})

# every exported entry point of include/cs3d.h
EXPORTS = [
    "cs3d_version", "cs3d_strerror", "cs3d_config_read_json", "cs3d_config_to_params", "cs3d_mesh_read",
    "cs3d_topology_build", "cs3d_rng_init", "cs3d_rng_draw", "cs3d_rng_random_vector", "cs3d_seed_map",
    "cs3d_initial_stiffness", "cs3d_init_positions", "cs3d_traj_open", "cs3d_traj_write_frame", "cs3d_traj_close", "cs3d_create",
    "cs3d_create_ensemble", "cs3d_load_state", "cs3d_set_rng", "cs3d_get_rng", "cs3d_step", "cs3d_get_state",
    "cs3d_get_forces", "cs3d_get_random_force", "cs3d_get_cells", "cs3d_get_grid", "cs3d_set_option", "cs3d_get_pairs",
    "cs3d_get_events", "cs3d_get_far_counts", "cs3d_volume_histogram", "cs3d_last_error", "cs3d_get_stats", "cs3d_profile_step", "cs3d_last_step_ms",
    "cs3d_destroy", "cs3d_forces_static", "cs3d_get_state_async", "cs3d_wait_state", "cs3d_host_alloc",
    "cs3d_host_free", "cs3d_set_skin_schedule",
]

_lib = None


class CS3DError(RuntimeError):
    def __init__(self, where, status, bits=0):
        self.status = status
        self.bits = bits
        msg = "%s: %s (%d)" % (where, lib().cs3d_strerror(status).decode(), status)
        if bits:
            msg += " bits=" + "|".join(v for k, v in ERRBITS.items() if bits & k)
        super().__init__(msg)


def lib():
    """The loaded libcs3d.so.  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libcs3d.so not built: run `python -m cellsim3d_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int32)
    L.cs3d_version.restype = C.c_int
    L.cs3d_strerror.restype = C.c_char_p
    L.cs3d_strerror.argtypes = [C.c_int]
    L.cs3d_config_read_json.argtypes = [C.c_char_p, C.POINTER(Config), C.c_char_p, C.c_int]
    L.cs3d_config_to_params.argtypes = [C.POINTER(Config), C.POINTER(Params)]
    L.cs3d_mesh_read.argtypes = [C.c_char_p, C.POINTER(Mesh)]
    L.cs3d_topology_build.argtypes = [C.POINTER(Mesh), fp, fp, fp, C.POINTER(Topology)]
    L.cs3d_rng_init.argtypes = [C.POINTER(Rng), C.c_int, C.c_int]
    L.cs3d_rng_draw.argtypes = [C.POINTER(Rng), fp, C.c_int]
    L.cs3d_rng_random_vector.argtypes = [C.POINTER(Rng), fp]
    L.cs3d_seed_map.argtypes = [C.c_int, ip, ip]
    L.cs3d_init_positions.argtypes = [C.POINTER(Config), C.POINTER(Mesh), C.c_int, C.POINTER(Rng), fp, fp, fp]
    L.cs3d_initial_stiffness.argtypes = [C.POINTER(Config), C.c_int, fp, fp, fp, C.POINTER(Rng), fp]
    L.cs3d_traj_open.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(P)]
    L.cs3d_traj_write_frame.argtypes = [P, C.c_int, C.c_int, C.c_int, fp, fp, fp, ip]
    L.cs3d_traj_close.argtypes = [P, C.c_int]
    L.cs3d_create.argtypes = [C.POINTER(Params), C.POINTER(Topology), C.c_int, C.c_int, P, C.POINTER(P)]
    L.cs3d_create_ensemble.argtypes = [C.c_int, C.POINTER(Params), C.POINTER(Topology), ip, C.c_int, P,
                                       C.POINTER(P)]
    L.cs3d_load_state.argtypes = [P, C.c_int, C.c_int, fp, fp, fp, fp, fp, fp, fp, fp]
    L.cs3d_set_rng.argtypes = [P, C.c_int, C.POINTER(Rng)]
    L.cs3d_get_rng.argtypes = [P, C.c_int, C.POINTER(Rng)]
    L.cs3d_step.argtypes = [P, C.c_int]
    L.cs3d_get_state.argtypes = [P, C.c_int, ip, fp, fp, fp, fp, fp, fp, fp, fp]
    L.cs3d_get_state_async.argtypes = [P, C.c_int, C.c_int, ip, fp, fp, fp, fp, fp, fp, fp, fp]
    L.cs3d_wait_state.argtypes = [P, C.c_int]
    L.cs3d_host_alloc.argtypes = [C.c_size_t, C.POINTER(C.c_void_p)]
    L.cs3d_host_free.argtypes = [C.c_void_p]
    L.cs3d_get_forces.argtypes = [P, C.c_int, fp, fp, fp, fp, fp, fp]
    L.cs3d_get_random_force.argtypes = [P, C.c_int, fp, fp, fp]
    L.cs3d_get_cells.argtypes = [P, C.c_int, fp, fp, fp, fp]
    L.cs3d_get_grid.argtypes = [P, C.c_int, fp, ip]
    L.cs3d_set_option.argtypes = [P, C.c_int, C.c_longlong]
    L.cs3d_set_skin_schedule.argtypes = [P, C.c_int, ip, fp]
    L.cs3d_get_pairs.argtypes = [P, C.c_int, C.c_int, ip, C.c_longlong, C.POINTER(C.c_longlong)]
    L.cs3d_get_events.argtypes = [P, C.c_int, ip, C.c_int, ip]
    L.cs3d_get_far_counts.argtypes = [P, C.c_int, ip, C.c_int, ip]
    L.cs3d_volume_histogram.argtypes = [P, C.c_int, C.c_float, C.c_float, C.c_int, C.POINTER(C.c_int64), fp]
    L.cs3d_last_error.argtypes = [P, C.c_int, C.POINTER(C.c_uint32)]
    L.cs3d_get_stats.argtypes = [P, C.POINTER(C.c_longlong), C.c_int]
    L.cs3d_profile_step.argtypes = [P, C.c_int, fp, C.c_char_p, C.c_int, C.c_int, ip]
    L.cs3d_last_step_ms.argtypes = [P, fp]
    L.cs3d_destroy.argtypes = [P]
    L.cs3d_forces_static.argtypes = [C.POINTER(Params), C.POINTER(Topology), C.c_int] + [C.c_void_p] * 14 + [P]
    for name in EXPORTS:
        fn = getattr(L, name)
        if name not in ("cs3d_strerror",):
            fn.restype = C.c_int
    _lib = L
    return L


def check(status, where):
    if status != OK:
        raise CS3DError(where, status)
    return status
