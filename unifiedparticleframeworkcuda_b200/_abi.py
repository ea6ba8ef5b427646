"""ctypes mirror of the C ABI declared in include/upf.h.

Layouts here must match the header field for field; tests/test_abi.py checks
the sizes against the compiled library.
"""
import ctypes as C

LUT_SIZE = 300
LUT_ENTRIES = 301
GRID_RESOLUTION = 1024

# particle types (ParticleObjectType, src/cpu/UnifiedParticle.h:14-23)
RIGID, SOFT, LIQUID, GRANULAR, CLOTH, SMOKE, FROZEN = range(7)

METHOD_WCSPH = 1
METHOD_PCISPH = 2

FLAG_WALL_WEIGHT = 1 << 0
FLAG_SURFACE_TENSION = 1 << 1
FLAG_PENALTY_WALLS = 1 << 2
FLAG_BOUNDARY_PRESSURE = 1 << 3
FLAG_ADHESION = 1 << 4
FLAG_RECORD_ITERATIONS = 1 << 5

STATUS = {
    0: "UPF_OK",
    1: "UPF_ERR_INVALID_ARG",
    2: "UPF_ERR_CUDA",
    3: "UPF_ERR_ALLOC",
    4: "UPF_ERR_NEIGHBOR_OVERFLOW",
    5: "UPF_ERR_NAN",
    6: "UPF_ERR_TIMEOUT",
    7: "UPF_ERR_STATE",
    8: "UPF_ERR_UNSUPPORTED",
    9: "UPF_ERR_NO_DEVICE",
    10: "UPF_ERR_IO",
}

F3 = C.c_float * 3


class UpfParams(C.Structure):
    _fields_ = [
        ("method", C.c_int32),
        ("flags", C.c_uint32),
        ("particle_spacing", C.c_float),
        ("particle_radius", C.c_float),
        ("support_radius", C.c_float),
        ("mass", C.c_float),
        ("rest_density", C.c_float),
        ("gas_constant", C.c_float),
        ("gamma", C.c_float),
        ("viscosity", C.c_float),
        ("gravity", C.c_float),
        ("dt", C.c_float),
        ("density_error_factor", C.c_float),
        ("density_error_fudge", C.c_float),
        ("max_density_error", C.c_float),
        ("min_loops", C.c_int32),
        ("max_loops", C.c_int32),
        ("surface_tension_gamma", C.c_float),
        ("surface_adhesion_beta", C.c_float),
        ("force_distance", C.c_float),
        ("max_boundary_force", C.c_float),
        ("spring_coefficient", C.c_float),
        ("spring_coefficient_boundary", C.c_float),
        ("damping_coefficient", C.c_float),
        ("terminal_speed", C.c_float),
        ("granular_kr", C.c_float),
        ("granular_kd", C.c_float),
        ("granular_kt", C.c_float),
        ("granular_mu", C.c_float),
        ("zindex_origin", F3),
        ("zindex_extent", F3),
        ("scales", F3),
        ("block_size", C.c_uint32),
        ("collision_min", F3),
        ("collision_max", F3),
        ("container_min", F3),
        ("container_max", F3),
        ("max_neighbors", C.c_uint32),
        ("search_cell", C.c_uint32),
        ("reserved", C.c_uint32 * 6),
    ]

    def copy(self):
        c = UpfParams()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(UpfParams))
        return c

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if hasattr(v, "__len__"):
                v = list(v)
            out[name] = v
        return out


class UpfStepStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("hit_max_loops", C.c_int32),
        ("max_predicted_density", C.c_float),
        ("density_error_percent", C.c_float),
        ("max_neighbor_count", C.c_uint32),
        ("error_flags", C.c_uint32),
        ("kinetic_energy", C.c_double),
        ("momentum", C.c_double * 3),
        ("iteration_max_density", C.c_float * 64),
        ("total_steps", C.c_int32),
        ("total_iterations", C.c_int32),
        ("steps_at_max_loops", C.c_int32),
        ("max_step_density_error_percent", C.c_float),
    ]


class UpfDeviceState(C.Structure):
    """upf_device_state: device pointers of a system's arrays."""
    _fields_ = [
        ("pos4", C.c_void_p), ("vel4", C.c_void_p), ("lag4", C.c_void_p), ("type", C.c_void_p), ("id", C.c_void_p),
        ("n", C.c_uint32), ("capacity_dynamic", C.c_uint32),
        ("sorted_pos4", C.c_void_p), ("sorted_id", C.c_void_p), ("predicted_pos4", C.c_void_p),
        ("pressure", C.c_void_p), ("pq4", C.c_void_p), ("density", C.c_void_p),
        ("loop_max_density_bits", C.c_void_p), ("stream", C.c_void_p),
    ]


class UpfPhaseTimes(C.Structure):
    _fields_ = [
        ("sort_ms", C.c_float),
        ("neighbors_ms", C.c_float),
        ("forces_ms", C.c_float),
        ("loop_ms", C.c_float),
        ("integrate_ms", C.c_float),
        ("density_ms_total", C.c_float),
        ("pforce_ms_total", C.c_float),
        ("iterations", C.c_int32),
        ("launches", C.c_int32),
    ]


class UpfLaunchConfig(C.Structure):
    """upf_launch_config (include/upf.h): launch shapes of the tunable passes."""
    _fields_ = [
        ("nlist_threads", C.c_int32),
        ("external_threads", C.c_int32),
        ("density_threads", C.c_int32),
        ("density_rows", C.c_int32),
        ("pforce_threads", C.c_int32),
        ("pforce_rows", C.c_int32),
        ("density_mode", C.c_int32),
        ("pforce_mode", C.c_int32),
        ("nlist_mode", C.c_int32),
        ("measured_ms", C.c_float * 4),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "measured_ms"}
        d["measured_ms"] = list(self.measured_ms)
        return d


class UpfAdjointOptions(C.Structure):
    """upf_adjoint_options (include/upf.h)."""
    _fields_ = [
        ("steps", C.c_int32),
        ("checkpoint_interval", C.c_int32),
        ("loop_iterations", C.c_int32),
        ("target", C.c_float * 3),
        ("com_weight", C.c_float),
        ("density_weight", C.c_float),
        ("density_smoothing", C.c_float),
    ]

