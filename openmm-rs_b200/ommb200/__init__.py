"""Python front end of the B200 engine, mirroring openmm-py's classes (System, NonbondedForce,
GBSAOBCForce, HarmonicBondForce, HarmonicAngleForce, LangevinMiddleIntegrator, Context, State;
crates/openmm-py/src/lib.rs, gbsa_obc.rs, integrators.rs) over the C ABI in include/ommb200.h.

There is no CPU fallback: if libommb200.so is missing or no CUDA device is present, the calls
that need it raise.  Errors of the C ABI become Python exceptions carrying its message.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libommb200.so"

OK = 0
ERR_INVALID_ARG = -1
ERR_CONSTRAINT = -2
ERR_NONFINITE = -3
ERR_NLIST_OVERFLOW = -4
ERR_TIMEOUT = -5
ERR_CUDA = -6
ERR_UNSUPPORTED = -7
ERR_OUT_OF_MEMORY = -8

PRECISION_MIXED = 0
PRECISION_DOUBLE = 1

STATE_POSITIONS, STATE_VELOCITIES, STATE_FORCES, STATE_ENERGY, STATE_VIRIAL = 1, 2, 4, 8, 16

NONBONDED_METHODS = {"NoCutoff": 0, "CutoffNonPeriodic": 1, "CutoffPeriodic": 2, "Ewald": 3,
                     "PME": 4, "LJPME": 5}


class OmmB200Error(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class InvalidArgument(OmmB200Error, ValueError):
    pass


class ConstraintError(OmmB200Error):
    pass


class NonfiniteError(OmmB200Error, FloatingPointError):
    """A position or velocity became nonfinite during the steps."""


class TimeoutError_(OmmB200Error, TimeoutError):
    """A tensor-core kernel gave up waiting for its MMAs (OMMB200_ERR_TIMEOUT)."""


class NeighborListOverflow(OmmB200Error):
    """The neighbour list could not hold the pairs and could not grow any further."""


_ERRORS = {ERR_INVALID_ARG: InvalidArgument, ERR_CONSTRAINT: ConstraintError,
           ERR_NONFINITE: NonfiniteError, ERR_TIMEOUT: TimeoutError_,
           ERR_NLIST_OVERFLOW: NeighborListOverflow}


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("use_cuda_graph", C.c_int),
                ("neighbor_skin", C.c_double), ("steps_per_graph", C.c_int),
                ("pme_bricks", C.c_int), ("prune_margin", C.c_double), ("pair_cull", C.c_int)]


class LearnedRadiiStats(C.Structure):
    _fields_ = [("judges", C.c_int64), ("learned_steps", C.c_int64), ("exact_steps", C.c_int64),
                ("active", C.c_int), ("last_radius_error", C.c_double), ("last_loss", C.c_double)]


class BarostatStats(C.Structure):
    _fields_ = [("attempted", C.c_uint64), ("accepted", C.c_uint64), ("volume_scale", C.c_double),
                ("last_accepted", C.c_int), ("last_old_volume", C.c_double),
                ("last_new_volume", C.c_double), ("last_energy_change", C.c_double),
                ("last_work", C.c_double), ("last_uniform", C.c_double)]


class StateInfo(C.Structure):
    _fields_ = [("time", C.c_double), ("step_count", C.c_int64),
                ("potential_energy", C.c_double), ("kinetic_energy", C.c_double),
                ("box", C.c_double * 9), ("virial", C.c_double * 9)]


_lib = None


def library() -> C.CDLL:
    """Load libommb200.so (built by `make -C openmm-rs_b200`); raises if it is missing."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            raise ImportError(f"{_LIB_PATH} is missing: build it with `make -C openmm-rs_b200` "
                              "(the engine has no CPU fallback)")
        lib = C.CDLL(str(_LIB_PATH))
        lib.ommb200_last_error.restype = C.c_char_p
        lib.ommb200_version.restype = C.c_char_p
        P = C.c_void_p
        D = C.c_double
        I = C.c_int
        sig = {
            "ommb200_system_add_particle": [P, D, C.POINTER(I)],
            "ommb200_system_add_constraint": [P, I, I, D, C.POINTER(I)],
            "ommb200_nonbonded_add_particle": [P, D, D, D, C.POINTER(I)],
            "ommb200_nonbonded_set_particle_parameters": [P, I, D, D, D],
            "ommb200_nonbonded_add_exception": [P, I, I, D, D, D, C.POINTER(I)],
            "ommb200_nonbonded_create_exceptions_from_bonds": [P, I, C.POINTER(I), D, D],
            "ommb200_nonbonded_set_cutoff_distance": [P, D],
            "ommb200_nonbonded_set_reaction_field_dielectric": [P, D],
            "ommb200_nonbonded_set_ewald_error_tolerance": [P, D],
            "ommb200_nonbonded_set_switching_distance": [P, D],
            "ommb200_nonbonded_set_pme_parameters": [P, D, I, I, I],
            "ommb200_gbsa_obc_add_particle": [P, D, D, D, C.POINTER(I)],
            "ommb200_gbsa_obc_set_particle_parameters": [P, I, D, D, D],
            "ommb200_gbsa_obc_set_cutoff_distance": [P, D],
            "ommb200_gbsa_obc_set_solvent_dielectric": [P, D],
            "ommb200_gbsa_obc_set_solute_dielectric": [P, D],
            "ommb200_gbsa_obc_set_surface_area_energy": [P, D],
            "ommb200_harmonic_bond_add_bond": [P, I, I, D, D, C.POINTER(I)],
            "ommb200_harmonic_angle_add_angle": [P, I, I, I, D, D, C.POINTER(I)],
            "ommb200_langevin_middle_create": [D, D, D, C.POINTER(P)],
            "ommb200_integrator_set_constraint_tolerance": [P, D],
            "ommb200_integrator_set_temperature": [P, D],
            "ommb200_integrator_set_friction": [P, D],
            "ommb200_integrator_set_step_size": [P, D],
            "ommb200_integrator_set_integration_force_groups": [P, C.c_uint32],
            "ommb200_context_create": [P, P, C.POINTER(Options), C.POINTER(P)],
            "ommb200_context_create_batch": [C.POINTER(P), I, P, C.POINTER(Options),
                                             C.POINTER(P)],
            "ommb200_context_num_systems": [P, C.POINTER(I)],
            "ommb200_context_system_range": [P, I, C.POINTER(I), C.POINTER(I)],
            "ommb200_context_get_system_energies": [P, C.c_uint32, C.POINTER(D), C.POINTER(D)],
            "ommb200_context_set_positions": [P, C.POINTER(D), I],
            "ommb200_context_set_velocities": [P, C.POINTER(D), I],
            "ommb200_context_set_velocities_to_temperature": [P, D, I],
            "ommb200_context_set_periodic_box_vectors": [P, C.POINTER(D), C.POINTER(D), C.POINTER(D)],
            "ommb200_context_set_time": [P, D],
            "ommb200_context_set_step_count": [P, C.c_int64],
            "ommb200_context_apply_constraints": [P, D],
            "ommb200_context_apply_velocity_constraints": [P, D],
            "ommb200_context_step": [P, I],
            "ommb200_context_get_tuning": [P, C.POINTER(D), C.POINTER(I), C.POINTER(I)],
            "ommb200_context_nlist_capacity": [P, C.POINTER(I), C.POINTER(I), C.POINTER(I)],
            "ommb200_set_tensor_core_wait_limit": [C.c_longlong],
            "ommb200_context_nlist_prune_stats": [P, C.POINTER(I), C.POINTER(C.c_int64),
                                                  C.POINTER(D)],
            "ommb200_context_get_pair_cull": [P, C.POINTER(I), C.POINTER(C.c_int64)],
            "ommb200_monte_carlo_barostat_create": [D, D, I, C.POINTER(P)],
            "ommb200_monte_carlo_barostat_set_default_pressure": [P, D],
            "ommb200_monte_carlo_barostat_get_default_pressure": [P, C.POINTER(D)],
            "ommb200_monte_carlo_barostat_set_default_temperature": [P, D],
            "ommb200_monte_carlo_barostat_get_default_temperature": [P, C.POINTER(D)],
            "ommb200_monte_carlo_barostat_set_frequency": [P, I],
            "ommb200_monte_carlo_barostat_get_frequency": [P, C.POINTER(I)],
            "ommb200_monte_carlo_barostat_set_scale_molecules_as_rigid": [P, I],
            "ommb200_monte_carlo_barostat_get_scale_molecules_as_rigid": [P, C.POINTER(I)],
            "ommb200_monte_carlo_barostat_set_random_number_seed": [P, I],
            "ommb200_monte_carlo_barostat_get_random_number_seed": [P, C.POINTER(I)],
            "ommb200_context_set_parameter": [P, C.c_char_p, D],
            "ommb200_context_get_parameter": [P, C.c_char_p, C.POINTER(D)],
            "ommb200_context_get_barostat_stats": [P, C.POINTER(BarostatStats)],
            "ommb200_context_get_state": [P, I, C.c_uint32, C.POINTER(D), C.POINTER(D),
                                          C.POINTER(D), C.POINTER(StateInfo)],
            "ommb200_context_get_pme_parameters": [P, C.POINTER(D), C.POINTER(I), C.POINTER(I),
                                                   C.POINTER(I)],
            "ommb200_context_get_pme_layout": [P, C.POINTER(I), C.POINTER(I)],
            "ommb200_context_debug_pair_list": [P, C.c_int64, C.POINTER(C.c_int32),
                                                C.POINTER(C.c_int64)],
            "ommb200_context_kernel_times": [P, I, C.c_char_p, I, C.POINTER(D), C.POINTER(I),
                                             C.POINTER(I)],
            "ommb200_radii_mlp_forward": [I, P, P, P, P, P],
            "ommb200_gbsa_obc_set_learned_radii": [P, I, I, D, I],
            "ommb200_context_update_nonbonded_parameters": [P, P],
            "ommb200_context_update_gbsa_obc_parameters": [P, P],
            "ommb200_context_checkpoint_size": [P, C.POINTER(C.c_int64)],
            "ommb200_context_create_checkpoint": [P, P, C.c_int64],
            "ommb200_context_load_checkpoint": [P, P, C.c_int64],
            "ommb200_context_get_learned_radii_stats": [P, C.POINTER(LearnedRadiiStats)],
            "ommb200_context_get_radii_mlp_params": [P, C.POINTER(C.c_float)],
            "ommb200_context_set_radii_mlp_params": [P, C.POINTER(C.c_float)],
            "ommb200_radii_mlp_train": [I, P, P, P, P, P, I, I, D, C.c_uint64, P, P, P],
        }
        for name, args in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = lib
    return _lib


def version() -> str:
    return library().ommb200_version().decode()


def measure_fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA throughput in TFLOP/s (FMA = 2 flops)."""
    v = C.c_double()
    _check(library().ommb200_measure_fp32_peak(device, C.byref(v)))
    return v.value


def _check(code: int) -> None:
    if code != OK:
        msg = library().ommb200_last_error().decode()
        raise _ERRORS.get(code, OmmB200Error)(code, msg)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _vec3(v) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(3))
    return a


# ---- System ------------------------------------------------------------------------------
class System:
    """system.rs:43-233.  Default periodic box: a 2 nm cube."""

    def __init__(self):
        h = C.c_void_p()
        _check(library().ommb200_system_create(C.byref(h)))
        self._h = h
        self._forces = []

    def _take(self):
        if self._h is None:
            raise InvalidArgument(ERR_INVALID_ARG, "System already moved into a Context")
        h, self._h = self._h, None
        return h

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.ommb200_system_destroy(self._h)
            self._h = None

    def add_particle(self, mass: float) -> int:
        i = C.c_int()
        _check(library().ommb200_system_add_particle(self._h, mass, C.byref(i)))
        return i.value

    def num_particles(self) -> int:
        i = C.c_int()
        _check(library().ommb200_system_num_particles(self._h, C.byref(i)))
        return i.value

    def add_constraint(self, particle1: int, particle2: int, distance: float) -> int:
        i = C.c_int()
        _check(library().ommb200_system_add_constraint(self._h, particle1, particle2, distance,
                                                       C.byref(i)))
        return i.value

    def set_default_periodic_box_vectors(self, a, b, c) -> None:
        va, vb, vc = _vec3(a), _vec3(b), _vec3(c)
        _check(library().ommb200_system_set_default_periodic_box_vectors(
            self._h, _dptr(va), _dptr(vb), _dptr(vc)))

    def add_force(self, force) -> int:
        i = C.c_int()
        _check(library().ommb200_system_add_force(self._h, force._h, C.byref(i)))
        force._owned = True
        self._forces.append(force)
        return i.value

    def num_forces(self) -> int:
        return len(self._forces)


class _Force:
    _create = None

    def __init__(self):
        h = C.c_void_p()
        _check(getattr(library(), self._create)(C.byref(h)))
        self._h = h
        self._owned = False

    def __del__(self):
        if getattr(self, "_h", None) is not None and not self._owned and _lib is not None:
            _lib.ommb200_force_destroy(self._h)

    def set_force_group(self, group: int) -> None:
        _check(library().ommb200_force_set_group(self._h, int(group)))

    def get_force_group(self) -> int:
        g = C.c_int()
        _check(library().ommb200_force_get_group(self._h, C.byref(g)))
        return g.value


class NonbondedForce(_Force):
    """forces/nonbonded.rs:122-658 (method names of openmm-py lib.rs:222-530)."""

    _create = "ommb200_nonbonded_create"

    def add_particle(self, charge: float, sigma: float, epsilon: float) -> int:
        i = C.c_int()
        _check(library().ommb200_nonbonded_add_particle(self._h, charge, sigma, epsilon, C.byref(i)))
        return i.value

    def set_particle_parameters(self, index, charge, sigma, epsilon) -> None:
        _check(library().ommb200_nonbonded_set_particle_parameters(self._h, index, charge, sigma, epsilon))

    def get_particle_parameters(self, index):
        q, s, e = C.c_double(), C.c_double(), C.c_double()
        _check(library().ommb200_nonbonded_get_particle_parameters(self._h, index, C.byref(q),
                                                                   C.byref(s), C.byref(e)))
        return q.value, s.value, e.value

    def num_particles(self) -> int:
        i = C.c_int()
        _check(library().ommb200_nonbonded_num_particles(self._h, C.byref(i)))
        return i.value

    def add_exception(self, particle1, particle2, charge_prod, sigma, epsilon) -> int:
        i = C.c_int()
        _check(library().ommb200_nonbonded_add_exception(self._h, particle1, particle2, charge_prod,
                                                         sigma, epsilon, C.byref(i)))
        return i.value

    def num_exceptions(self) -> int:
        i = C.c_int()
        _check(library().ommb200_nonbonded_num_exceptions(self._h, C.byref(i)))
        return i.value

    def create_exceptions_from_bonds(self, bonds, coulomb14scale, lj14scale) -> None:
        b = np.ascontiguousarray(np.asarray(bonds, dtype=np.int32).reshape(-1))
        _check(library().ommb200_nonbonded_create_exceptions_from_bonds(
            self._h, len(b) // 2, b.ctypes.data_as(C.POINTER(C.c_int)), coulomb14scale, lj14scale))

    def set_nonbonded_method(self, method) -> None:
        m = NONBONDED_METHODS[method] if isinstance(method, str) else int(method)
        _check(library().ommb200_nonbonded_set_method(self._h, m))

    def set_cutoff_distance(self, cutoff: float) -> None:
        _check(library().ommb200_nonbonded_set_cutoff_distance(self._h, cutoff))

    def set_reaction_field_dielectric(self, eps: float) -> None:
        _check(library().ommb200_nonbonded_set_reaction_field_dielectric(self._h, eps))

    def set_ewald_error_tolerance(self, tol: float) -> None:
        _check(library().ommb200_nonbonded_set_ewald_error_tolerance(self._h, tol))

    def set_use_dispersion_correction(self, enabled: bool) -> None:
        _check(library().ommb200_nonbonded_set_use_dispersion_correction(self._h, int(enabled)))

    def set_use_switching_function(self, enabled: bool) -> None:
        _check(library().ommb200_nonbonded_set_use_switching_function(self._h, int(enabled)))

    def set_switching_distance(self, distance: float) -> None:
        _check(library().ommb200_nonbonded_set_switching_distance(self._h, distance))

    def set_exceptions_use_periodic_boundary_conditions(self, enabled: bool) -> None:
        _check(library().ommb200_nonbonded_set_exceptions_use_periodic_boundary_conditions(
            self._h, int(enabled)))

    def set_pme_parameters(self, alpha, nx, ny, nz) -> None:
        _check(library().ommb200_nonbonded_set_pme_parameters(self._h, alpha, nx, ny, nz))

    def set_reciprocal_space_force_group(self, group: int) -> None:
        _check(library().ommb200_nonbonded_set_reciprocal_space_force_group(self._h, group))

    def set_include_direct_space(self, enabled: bool) -> None:
        _check(library().ommb200_nonbonded_set_include_direct_space(self._h, int(enabled)))


class GBSAOBCForce(_Force):
    """forces/gbsa_obc.rs:61-133 (openmm-py gbsa_obc.rs)."""

    _create = "ommb200_gbsa_obc_create"

    def add_particle(self, charge, radius, scaling_factor) -> int:
        i = C.c_int()
        _check(library().ommb200_gbsa_obc_add_particle(self._h, charge, radius, scaling_factor,
                                                       C.byref(i)))
        return i.value

    def set_particle_parameters(self, index, charge, radius, scaling_factor) -> None:
        _check(library().ommb200_gbsa_obc_set_particle_parameters(self._h, index, charge, radius,
                                                                  scaling_factor))

    def set_nonbonded_method(self, method: int) -> None:
        _check(library().ommb200_gbsa_obc_set_method(self._h, int(method)))

    def set_learned_radii(self, enabled: bool = True, judge_interval: int = 50,
                          radius_tolerance: float = 0.01, train_steps: int = 10) -> None:
        """Replace the O(N^2) descreening passes by a short-range integral plus a network
        tail, judged (and trained) against the exact pass every `judge_interval` steps."""
        _check(library().ommb200_gbsa_obc_set_learned_radii(self._h, int(enabled),
                                                            int(judge_interval),
                                                            float(radius_tolerance),
                                                            int(train_steps)))

    def set_cutoff_distance(self, value) -> None:
        _check(library().ommb200_gbsa_obc_set_cutoff_distance(self._h, value))

    def set_solvent_dielectric(self, value) -> None:
        _check(library().ommb200_gbsa_obc_set_solvent_dielectric(self._h, value))

    def set_solute_dielectric(self, value) -> None:
        _check(library().ommb200_gbsa_obc_set_solute_dielectric(self._h, value))

    def set_surface_area_energy(self, value) -> None:
        _check(library().ommb200_gbsa_obc_set_surface_area_energy(self._h, value))


class HarmonicBondForce(_Force):
    _create = "ommb200_harmonic_bond_create"

    def add_bond(self, particle1, particle2, length, k) -> int:
        i = C.c_int()
        _check(library().ommb200_harmonic_bond_add_bond(self._h, particle1, particle2, length, k,
                                                        C.byref(i)))
        return i.value

    def set_uses_periodic_boundary_conditions(self, use_pbc: bool) -> None:
        _check(library().ommb200_harmonic_bond_set_uses_pbc(self._h, int(use_pbc)))


class MonteCarloBarostat(_Force):
    """forces/barostat.rs:44-119 (openmm-py barostat.rs): isotropic Monte Carlo volume moves
    every `frequency` steps at `pressure` (bar) and `temperature` (K)."""

    def __init__(self, pressure: float = 1.0, temperature: float = 300.0, frequency: int = 25):
        h = C.c_void_p()
        _check(library().ommb200_monte_carlo_barostat_create(float(pressure), float(temperature),
                                                             int(frequency), C.byref(h)))
        self._h = h
        self._owned = False

    PRESSURE = "MonteCarloPressure"
    TEMPERATURE = "MonteCarloTemperature"

    def _get(self, name, ctype):
        v = ctype()
        _check(getattr(library(), f"ommb200_monte_carlo_barostat_get_{name}")(self._h, C.byref(v)))
        return v.value

    def set_default_pressure(self, pressure: float) -> None:
        _check(library().ommb200_monte_carlo_barostat_set_default_pressure(self._h, float(pressure)))

    def get_default_pressure(self) -> float:
        return self._get("default_pressure", C.c_double)

    def set_default_temperature(self, temperature: float) -> None:
        _check(library().ommb200_monte_carlo_barostat_set_default_temperature(self._h,
                                                                              float(temperature)))

    def get_default_temperature(self) -> float:
        return self._get("default_temperature", C.c_double)

    def set_frequency(self, frequency: int) -> None:
        """Reaches the Contexts that already hold this barostat, as in the reference."""
        _check(library().ommb200_monte_carlo_barostat_set_frequency(self._h, int(frequency)))

    def get_frequency(self) -> int:
        return self._get("frequency", C.c_int)

    def set_scale_molecules_as_rigid(self, rigid: bool) -> None:
        """Taken by a Context when it is created; later changes do not reach it."""
        _check(library().ommb200_monte_carlo_barostat_set_scale_molecules_as_rigid(self._h,
                                                                                   int(rigid)))

    def get_scale_molecules_as_rigid(self) -> bool:
        return bool(self._get("scale_molecules_as_rigid", C.c_int))

    def set_random_number_seed(self, seed: int) -> None:
        _check(library().ommb200_monte_carlo_barostat_set_random_number_seed(self._h, int(seed)))

    def get_random_number_seed(self) -> int:
        return self._get("random_number_seed", C.c_int)


class HarmonicAngleForce(_Force):
    _create = "ommb200_harmonic_angle_create"

    def add_angle(self, particle1, particle2, particle3, angle, k) -> int:
        i = C.c_int()
        _check(library().ommb200_harmonic_angle_add_angle(self._h, particle1, particle2, particle3,
                                                          angle, k, C.byref(i)))
        return i.value

    def set_uses_periodic_boundary_conditions(self, use_pbc: bool) -> None:
        _check(library().ommb200_harmonic_angle_set_uses_pbc(self._h, int(use_pbc)))


class LangevinMiddleIntegrator:
    """integrators/langevin.rs:14-102: temperature (K), friction (1/ps), step size (ps)."""

    def __init__(self, temperature: float, friction: float, step_size: float):
        h = C.c_void_p()
        _check(library().ommb200_langevin_middle_create(temperature, friction, step_size, C.byref(h)))
        self._h = h
        self.step_size = step_size

    def _take(self):
        if self._h is None:
            raise InvalidArgument(ERR_INVALID_ARG, "integrator already moved into a Context")
        h, self._h = self._h, None
        return h

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.ommb200_integrator_destroy(self._h)

    def set_random_number_seed(self, seed: int) -> None:
        _check(library().ommb200_integrator_set_random_number_seed(self._h, int(seed)))

    def set_constraint_tolerance(self, tol: float) -> None:
        _check(library().ommb200_integrator_set_constraint_tolerance(self._h, tol))

    def set_temperature(self, t: float) -> None:
        _check(library().ommb200_integrator_set_temperature(self._h, t))

    def set_friction(self, f: float) -> None:
        _check(library().ommb200_integrator_set_friction(self._h, f))

    def set_step_size(self, dt: float) -> None:
        _check(library().ommb200_integrator_set_step_size(self._h, dt))
        self.step_size = dt

    def set_integration_force_groups(self, groups: int) -> None:
        _check(library().ommb200_integrator_set_integration_force_groups(self._h, groups & 0xFFFFFFFF))


class State:
    """state.rs:47-58 plus the virial."""

    def __init__(self, info: StateInfo, positions, velocities, forces, energy: bool, virial: bool):
        self.time = info.time
        self.step_count = info.step_count
        self.positions = positions
        self.velocities = velocities
        self.forces = forces
        self.potential_energy = info.potential_energy if energy else None
        self.kinetic_energy = info.kinetic_energy
        self.periodic_box_vectors = np.array(info.box).reshape(3, 3)
        self.virial = np.array(info.virial).reshape(3, 3) if virial else None

    def get_positions(self):
        return self.positions

    def get_velocities(self):
        return self.velocities

    def get_forces(self):
        return self.forces

    def get_potential_energy(self):
        return self.potential_energy

    def get_kinetic_energy(self):
        return self.kinetic_energy


def _options(precision, device, use_cuda_graph, neighbor_skin, steps_per_graph,
             pme_bricks=-1, prune_margin=-1.0, pair_cull=-1) -> "Options":
    opt = Options()
    opt.precision = {"mixed": PRECISION_MIXED, "double": PRECISION_DOUBLE}[precision]
    opt.device = device
    opt.use_cuda_graph = int(use_cuda_graph)
    opt.neighbor_skin = neighbor_skin
    opt.steps_per_graph = steps_per_graph
    opt.pme_bricks = pme_bricks
    opt.prune_margin = prune_margin
    opt.pair_cull = pair_cull
    return opt


class Context:
    """context.rs:83-1163.  Takes ownership of `system` and `integrator` (context.rs:83-87)."""

    def __init__(self, system: System, integrator: LangevinMiddleIntegrator, precision="mixed",
                 device: int = 0, use_cuda_graph: bool = True, neighbor_skin: float = 0.0,
                 steps_per_graph: int = 0, pme_bricks: int = -1, prune_margin: float = -1.0,
                 pair_cull: int = -1):
        """`pme_bricks`: brick-owned PME gather in rectangular periodic boxes, -1 when
        the grid has at least two bricks per SM, 0 never, 1 whenever the box allows (the forces
        are the same either way).  `prune_margin` (nm): the pruned pair list between rebuilds
        (0 off, < 0 the default: off until `autotune` picks a margin).  `pair_cull`: tiles per
        warp run of the culling pair kernel, which drops entries beyond the cutoff of their half
        block at every evaluation (0 off, < 0 the default)."""
        n = system.num_particles()
        opt = _options(precision, device, use_cuda_graph, neighbor_skin, steps_per_graph,
                       pme_bricks, prune_margin, pair_cull)
        h = C.c_void_p()
        sys_h, int_h = system._take(), integrator._take()
        _check(library().ommb200_context_create(sys_h, int_h, C.byref(opt), C.byref(h)))
        self._h = h
        self._n = n
        self.step_size = integrator.step_size
        self.precision = precision

    def __del__(self):
        self.close()

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.ommb200_context_destroy(self._h)
            self._h = None

    def num_particles(self) -> int:
        return self._n

    def _arr(self, values) -> np.ndarray:
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(self._n, 3))
        return a

    def set_positions(self, positions) -> None:
        a = self._arr(positions)
        _check(library().ommb200_context_set_positions(self._h, _dptr(a), self._n))

    def set_velocities(self, velocities) -> None:
        a = self._arr(velocities)
        _check(library().ommb200_context_set_velocities(self._h, _dptr(a), self._n))

    def set_velocities_to_temperature(self, temperature: float, seed: int = 0) -> None:
        _check(library().ommb200_context_set_velocities_to_temperature(self._h, temperature, seed))

    def set_periodic_box_vectors(self, a, b, c) -> None:
        va, vb, vc = _vec3(a), _vec3(b), _vec3(c)
        _check(library().ommb200_context_set_periodic_box_vectors(self._h, _dptr(va), _dptr(vb),
                                                                  _dptr(vc)))

    def set_time(self, time: float) -> None:
        _check(library().ommb200_context_set_time(self._h, time))

    def set_step_count(self, steps: int) -> None:
        _check(library().ommb200_context_set_step_count(self._h, steps))

    def apply_constraints(self, tolerance: float) -> None:
        _check(library().ommb200_context_apply_constraints(self._h, tolerance))

    def apply_velocity_constraints(self, tolerance: float) -> None:
        _check(library().ommb200_context_apply_velocity_constraints(self._h, tolerance))

    def step(self, steps: int) -> None:
        _check(library().ommb200_context_step(self._h, int(steps)))

    def set_parameter(self, name: str, value: float) -> None:
        """context.rs:251-261: a global parameter of the System's forces."""
        _check(library().ommb200_context_set_parameter(self._h, name.encode(), float(value)))

    def get_parameter(self, name: str) -> float:
        v = C.c_double()
        _check(library().ommb200_context_get_parameter(self._h, name.encode(), C.byref(v)))
        return v.value

    def barostat_stats(self) -> dict:
        """Attempted / accepted volume moves, the current volume step and the last move."""
        st = BarostatStats()
        _check(library().ommb200_context_get_barostat_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in BarostatStats._fields_}

    def get_state(self, positions=False, velocities=False, forces=False, energy=False,
                  virial=False, groups=-1) -> State:
        flags = ((STATE_POSITIONS if positions else 0) | (STATE_VELOCITIES if velocities else 0) |
                 (STATE_FORCES if forces else 0) | (STATE_ENERGY if energy else 0) |
                 (STATE_VIRIAL if virial else 0))
        p = np.zeros((self._n, 3)) if positions else None
        v = np.zeros((self._n, 3)) if velocities else None
        f = np.zeros((self._n, 3)) if forces else None
        info = StateInfo()
        null = C.POINTER(C.c_double)()
        _check(library().ommb200_context_get_state(
            self._h, flags, groups & 0xFFFFFFFF, _dptr(p) if p is not None else null,
            _dptr(v) if v is not None else null, _dptr(f) if f is not None else null,
            C.byref(info)))
        return State(info, p, v, f, energy, virial)

    def get_pme_parameters(self):
        a, nx, ny, nz = C.c_double(), C.c_int(), C.c_int(), C.c_int()
        _check(library().ommb200_context_get_pme_parameters(self._h, C.byref(a), C.byref(nx),
                                                            C.byref(ny), C.byref(nz)))
        return a.value, (nx.value, ny.value, nz.value)

    def pme_layout(self) -> dict:
        """PME gather form: brick-owned (`bricks_in_use`) or eight lanes per particle; grid
        bricks."""
        u, n = C.c_int(), C.c_int()
        _check(library().ommb200_context_get_pme_layout(self._h, C.byref(u), C.byref(n)))
        return {"bricks_in_use": bool(u.value), "bricks": n.value}

    def debug_pair_list(self, max_pairs: int | None = None) -> np.ndarray:
        """The interacting nonbonded pairs (i < j) as evaluated by the pair kernel."""
        count = C.c_int64()
        _check(library().ommb200_context_debug_pair_list(self._h, 0, None, C.byref(count)))
        cap = count.value if max_pairs is None else max_pairs
        out = np.zeros((max(cap, 1), 2), dtype=np.int32)
        _check(library().ommb200_context_debug_pair_list(
            self._h, cap, out.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(count)))
        return out[:min(cap, count.value)]

    def update_nonbonded_parameters(self, force: "NonbondedForce") -> None:
        """context.rs:689-705: take the particle and exception parameters of `force` (which
        the caller keeps)."""
        _check(library().ommb200_context_update_nonbonded_parameters(self._h, force._h))

    def update_gbsa_obc_parameters(self, force: "GBSAOBCForce") -> None:
        """context.rs:680-687: take the charges, radii and scale factors of `force`."""
        _check(library().ommb200_context_update_gbsa_obc_parameters(self._h, force._h))

    def create_checkpoint(self) -> bytes:
        """The complete dynamic state (random stream included) as bytes."""
        n = C.c_int64()
        _check(library().ommb200_context_checkpoint_size(self._h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(library().ommb200_context_create_checkpoint(self._h, buf, n.value))
        return buf.raw

    def load_checkpoint(self, data: bytes) -> None:
        buf = C.create_string_buffer(bytes(data), len(data))
        _check(library().ommb200_context_load_checkpoint(self._h, buf, len(data)))

    def learned_radii_stats(self) -> dict:
        st = LearnedRadiiStats()
        _check(library().ommb200_context_get_learned_radii_stats(self._h, C.byref(st)))
        return {"judges": st.judges, "learned_steps": st.learned_steps,
                "exact_steps": st.exact_steps, "active": bool(st.active),
                "last_radius_error": st.last_radius_error, "last_loss": st.last_loss}

    def get_radii_mlp_params(self) -> np.ndarray:
        p = np.zeros(RADII_MLP_PARAMS, dtype=np.float32)
        _check(library().ommb200_context_get_radii_mlp_params(
            self._h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    def set_radii_mlp_params(self, params) -> None:
        """Install network parameters (normalisation included); trusted until the next judge."""
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float32).reshape(RADII_MLP_PARAMS))
        _check(library().ommb200_context_set_radii_mlp_params(
            self._h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def count_pairs(self) -> int:
        """Number of interacting nonbonded pairs at the current positions (pair kernel)."""
        count = C.c_int64()
        _check(library().ommb200_context_debug_pair_list(self._h, 0, None, C.byref(count)))
        return count.value

    def set_profiling(self, enabled: bool) -> None:
        _check(library().ommb200_context_set_profiling(self._h, int(enabled)))

    def autotune(self, trial_steps: int = 200) -> dict:
        """Pick the Verlet skin, tile width, pruned-list margin and pair-kernel grid by timing
        `trial_steps` MD steps per candidate; the state is restored afterwards."""
        skin, ctas, ms = C.c_double(), C.c_int(), C.c_double()
        _check(library().ommb200_context_autotune(self._h, int(trial_steps), C.byref(skin),
                                                  C.byref(ctas), C.byref(ms)))
        out = {"skin_nm": skin.value, "pair_ctas_per_sm": ctas.value, "ms_per_step": ms.value}
        out["tile_entries"] = self.tuning()["tile_entries"]
        out["prune_margin_nm"] = self.nlist_prune_stats()["margin_nm"]
        out["cull_tiles"] = self.tuning()["cull_tiles"]
        return out

    def tuning(self) -> dict:
        """Current skin, pair-kernel CTAs per SM, neighbour entries per i-group and tiles per
        warp run of the culling pair kernel (0: off)."""
        skin, ctas, width = C.c_double(), C.c_int(), C.c_int()
        _check(library().ommb200_context_get_tuning(self._h, C.byref(skin), C.byref(ctas),
                                                    C.byref(width)))
        return {"skin_nm": skin.value, "pair_ctas_per_sm": ctas.value,
                "tile_entries": width.value, "cull_tiles": self.pair_cull_stats()["cull_tiles"]}

    def pair_cull_stats(self) -> dict:
        """Culling pair kernel: tiles per warp run (0: not in use) and the rounds it has run
        so far, each 2 x 16 x 16 pair slots."""
        t, r = C.c_int(), C.c_int64()
        _check(library().ommb200_context_get_pair_cull(self._h, C.byref(t), C.byref(r)))
        return {"cull_tiles": t.value, "rounds": r.value}

    def nlist_stats(self) -> dict:
        """Neighbour-list state: tiles the pair kernel evaluates, blocks and masked tiles in
        use, rebuilds so far."""
        t, b, m, r = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
        _check(library().ommb200_context_nlist_stats(self._h, C.byref(t), C.byref(b), C.byref(m),
                                                     C.byref(r)))
        return {"tiles": t.value, "blocks": b.value, "masked_tiles": m.value,
                "rebuilds": r.value}

    def nlist_prune_stats(self) -> dict:
        """Pruned pair list: the last rebuild's tiles, prunes so far, margin (nm; 0 = the pair
        kernel reads the rebuild's tiles)."""
        t, c, m = C.c_int(), C.c_int64(), C.c_double()
        _check(library().ommb200_context_nlist_prune_stats(self._h, C.byref(t), C.byref(c),
                                                           C.byref(m)))
        return {"rebuild_tiles": t.value, "prunes": c.value, "margin_nm": m.value}

    def nlist_capacity(self) -> dict:
        """Neighbour-list capacities: tile slots, particles per x-y column, and how many times
        an overflow made them grow."""
        t, c, g = C.c_int(), C.c_int(), C.c_int()
        _check(library().ommb200_context_nlist_capacity(self._h, C.byref(t), C.byref(c),
                                                        C.byref(g)))
        return {"tile_capacity": t.value, "column_capacity": c.value, "regrows": g.value}

    def stream_handle(self) -> int:
        """cudaStream_t (as an integer) that every kernel of this Context runs on."""
        s = C.c_void_p()
        _check(library().ommb200_context_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def set_positions_from_pointer(self, host_ptr: int) -> None:
        """set_positions from a host buffer of 3N doubles (e.g. pinned memory)."""
        _check(library().ommb200_context_set_positions(
            self._h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double)), self._n))

    def set_velocities_from_pointer(self, host_ptr: int) -> None:
        _check(library().ommb200_context_set_velocities(
            self._h, C.cast(C.c_void_p(host_ptr), C.POINTER(C.c_double)), self._n))

    def get_state_into(self, pos_ptr: int, vel_ptr: int, energy: bool = True):
        """getState writing positions / velocities into caller buffers (3N doubles each);
        returns (potential energy or None, kinetic energy)."""
        flags = STATE_POSITIONS | STATE_VELOCITIES | (STATE_ENERGY if energy else 0)
        info = StateInfo()
        dp = C.POINTER(C.c_double)
        _check(library().ommb200_context_get_state(
            self._h, flags, 0xFFFFFFFF, C.cast(C.c_void_p(pos_ptr), dp),
            C.cast(C.c_void_p(vel_ptr), dp), dp(), C.byref(info)))
        return (info.potential_energy if energy else None), info.kinetic_energy

    def kernel_times(self):
        """{kernel name: (total ms, launches)} accumulated while profiling was enabled."""
        count = C.c_int()
        ms = (C.c_double * 64)()
        launches = (C.c_int * 64)()
        names = C.create_string_buffer(4096)
        _check(library().ommb200_context_kernel_times(self._h, 64, names, 4096, ms, launches,
                                                      C.byref(count)))
        keys = names.value.decode().split(";") if count.value else []
        return {k: (ms[i], launches[i]) for i, k in enumerate(keys)}


class BatchContext(Context):
    """Many independent Systems advanced by one Context (no reference counterpart: the
    reference runs one Context per System).  The Systems share their force kinds and global
    settings and, when there are several, are non-periodic; particle counts may differ.
    Positions, velocities and forces are the Systems' particles concatenated in order;
    `split` cuts such an array back into per-System pieces.  Takes ownership of every System
    and the integrator."""

    def __init__(self, systems, integrator: LangevinMiddleIntegrator, precision="mixed",
                 device: int = 0, use_cuda_graph: bool = True, neighbor_skin: float = 0.0,
                 steps_per_graph: int = 0):
        systems = list(systems)
        n = sum(s.num_particles() for s in systems)
        opt = _options(precision, device, use_cuda_graph, neighbor_skin, steps_per_graph)
        handles = (C.c_void_p * len(systems))(*[s._take() for s in systems])
        h = C.c_void_p()
        _check(library().ommb200_context_create_batch(handles, len(systems), integrator._take(),
                                                      C.byref(opt), C.byref(h)))
        self._h = h
        self._n = n
        self.step_size = integrator.step_size
        self.precision = precision
        self._ranges = [self.system_range(k) for k in range(self.num_systems())]

    def num_systems(self) -> int:
        out = C.c_int()
        _check(library().ommb200_context_num_systems(self._h, C.byref(out)))
        return out.value

    def system_range(self, index: int) -> tuple:
        """(first particle, particle count) of System `index`."""
        first, count = C.c_int(), C.c_int()
        _check(library().ommb200_context_system_range(self._h, index, C.byref(first),
                                                      C.byref(count)))
        return first.value, count.value

    def split(self, array) -> list:
        a = np.asarray(array)
        return [a[f:f + c] for f, c in self._ranges]

    def system_energies(self, groups: int = -1) -> tuple:
        """(potential, kinetic) energies of every System, kJ/mol, as two arrays."""
        k = len(self._ranges)
        pot, kin = np.zeros(k), np.zeros(k)
        _check(library().ommb200_context_get_system_energies(self._h, groups & 0xffffffff,
                                                             _dptr(pot), _dptr(kin)))
        return pot, kin


# ---- learned Born radii network (no reference counterpart) --------------------------------
RADII_MLP_PARAMS = 6403
RADII_MLP_TRAINABLE = 6337


def _devptr(t):
    if t is None:
        return None
    if not (t.is_cuda and t.is_contiguous() and str(t.dtype) in ("torch.float32", "torch.int32")):
        raise InvalidArgument(ERR_INVALID_ARG, "expected a contiguous float32/int32 CUDA tensor")
    return t.data_ptr()


def _stream_of(t):
    import torch

    return torch.cuda.current_stream(t.device).cuda_stream


def set_tensor_core_wait_limit(polls: int) -> None:
    """Polls after which the tensor-core kernels give up waiting for their MMAs (a diagnostic
    for the time-out path); polls < 0 restores the default."""
    _check(library().ommb200_set_tensor_core_wait_limit(int(polls)))


def radii_mlp_forward(features, params, with_gradient=True):
    """Network tail [n] and d tail / d features [n, 32] (None without `with_gradient`) for
    float32 CUDA tensors features [n, 32] and params [RADII_MLP_PARAMS]."""
    import torch

    n = int(features.shape[0])
    tail = torch.empty(n, dtype=torch.float32, device=features.device)
    dt = torch.empty(n, 32, dtype=torch.float32, device=features.device) if with_gradient else None
    _check(library().ommb200_radii_mlp_forward(n, _devptr(features), _devptr(params),
                                               _devptr(tail), _devptr(dt),
                                               _stream_of(features)))
    return tail, dt


def radii_mlp_train(features, targets, params, moments, step, steps, batch, learning_rate=1e-3,
                    seed=0, with_gradient=False):
    """Adam steps on the network, in place on params [RADII_MLP_PARAMS], moments
    [2, RADII_MLP_TRAINABLE] and step (int32 [1]); returns (losses [steps], last gradient or
    None)."""
    import torch

    n = int(features.shape[0])
    loss = torch.zeros(steps, dtype=torch.float32, device=features.device)
    grad = (torch.zeros(RADII_MLP_TRAINABLE, dtype=torch.float32, device=features.device)
            if with_gradient else None)
    _check(library().ommb200_radii_mlp_train(
        n, _devptr(features), _devptr(targets), _devptr(params), _devptr(moments), _devptr(step),
        steps, batch, learning_rate, seed, _devptr(grad), _devptr(loss), _stream_of(features)))
    return loss, grad
