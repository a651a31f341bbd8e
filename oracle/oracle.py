"""ctypes front end of the f64 CPU oracle (oracle/liboracle.so) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm import this module; the
product (openmm-rs_b200/) never does.  Each wrapper names the reference routine it restates
(paths relative to mogura-rs/openmm-rs/crates/openmm-core/src).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = _HERE / "liboracle.so"

NO_CUTOFF, CUTOFF_NONPERIODIC, CUTOFF_PERIODIC, EWALD, PME = 0, 1, 2, 3, 4
METHODS = {"NoCutoff": 0, "CutoffNonPeriodic": 1, "CutoffPeriodic": 2, "Ewald": 3, "PME": 4}


class NonbondedOptions(C.Structure):
    _fields_ = [
        ("method", C.c_int),
        ("cutoff", C.c_double),
        ("ewald_tolerance", C.c_double),
        ("reaction_field_dielectric", C.c_double),
        ("use_switching", C.c_int),
        ("switching_distance", C.c_double),
        ("use_dispersion_correction", C.c_int),
        ("exceptions_use_pbc", C.c_int),
        ("use_neighbor_cells", C.c_int),
        ("pme_alpha", C.c_double),
        ("pme_grid", C.c_int * 3),
        ("include_direct", C.c_int),
        ("include_reciprocal", C.c_int),
    ]


def build() -> None:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            build()
        _lib = C.CDLL(str(_LIB))
        D = C.POINTER(C.c_double)
        I = C.POINTER(C.c_int)
        _lib.orc_nonbonded.restype = C.c_int
        _lib.orc_pme_reciprocal.restype = C.c_double
        _lib.orc_ewald_reciprocal.restype = C.c_double
        _lib.orc_dispersion_coefficient.restype = C.c_double
        _lib.orc_dispersion_coefficient.argtypes = [C.c_int, D, D, C.c_double, C.c_int, C.c_double]
        _lib.orc_pair_set.restype = C.c_int64
        _lib.orc_pair_set.argtypes = [C.c_int, D, C.c_double, D, C.c_int, C.c_int, I, I, C.c_int,
                                      C.c_int64, C.POINTER(C.c_int32)]
        _lib.orc_gbsa_obc.restype = C.c_int
        _lib.orc_harmonic_bond.restype = C.c_double
        _lib.orc_harmonic_angle.restype = C.c_double
        _lib.orc_gaussian_noise.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, D]
        _lib.orc_constraints_solve.restype = C.c_int
        _lib.orc_settle_positions.restype = C.c_int
        _lib.orc_settle_positions.argtypes = [C.c_int, I, C.c_double, C.c_double, D, D, D]
        _lib.orc_settle_velocities.restype = C.c_int
        _lib.orc_lfmiddle_step.restype = C.c_int
        _lib.orc_lfmiddle_step.argtypes = [C.c_int, D, D, D, D, C.c_double, C.c_double, C.c_double,
                                           D, C.c_int, I, I, D, C.c_double, C.c_int, C.c_int, I,
                                           C.c_double, C.c_double]
        _lib.orc_kinetic_energy.restype = C.c_double
        _lib.orc_wtime.restype = C.c_double
        _lib.orc_max_threads.restype = C.c_int
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int))


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if shape is not None:
        a = a.reshape(shape)
    return a


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def pme_parameters(cutoff, tolerance, box):
    """nonbonded.rs:647-658 -> (alpha, (nx, ny, nz))."""
    alpha = C.c_double()
    dims = (C.c_int * 3)()
    lib().orc_pme_parameters(C.c_double(cutoff), C.c_double(tolerance), _d(_f64(box, (9,))),
                             C.byref(alpha), dims)
    return alpha.value, tuple(dims)


def nonbonded(pos, charge, sigma, epsilon, exceptions=(), method="PME", cutoff=1.0,
              ewald_tolerance=5e-4, box=None, use_switching=False, switching_distance=-1.0,
              use_dispersion_correction=True, exceptions_use_pbc=False, use_neighbor_cells=True,
              reaction_field_dielectric=78.3, pme=None, include_direct=True,
              include_reciprocal=True, threads=1, virial=False):
    """NonbondedForce::evaluate (nonbonded.rs:771-1042).  exceptions: (i, j, qq, sigma, eps).

    Returns (forces[N,3], energy) or (forces, energy, virial[3,3])."""
    pos = _f64(pos, (-1, 3))
    n = pos.shape[0]
    q, s, e = _f64(charge), _f64(sigma), _f64(epsilon)
    ex = list(exceptions)
    ei = _i32([x[0] for x in ex]) if ex else np.zeros(1, np.int32)
    ej = _i32([x[1] for x in ex]) if ex else np.zeros(1, np.int32)
    eqq = _f64([x[2] for x in ex]) if ex else np.zeros(1)
    es = _f64([x[3] for x in ex]) if ex else np.zeros(1)
    ee = _f64([x[4] for x in ex]) if ex else np.zeros(1)
    opt = NonbondedOptions()
    opt.method = METHODS[method] if isinstance(method, str) else int(method)
    opt.cutoff = cutoff
    opt.ewald_tolerance = ewald_tolerance
    opt.reaction_field_dielectric = reaction_field_dielectric
    opt.use_switching = int(use_switching)
    opt.switching_distance = switching_distance
    opt.use_dispersion_correction = int(use_dispersion_correction)
    opt.exceptions_use_pbc = int(exceptions_use_pbc)
    opt.use_neighbor_cells = int(use_neighbor_cells)
    if pme is not None:
        opt.pme_alpha = pme[0]
        for k in range(3):
            opt.pme_grid[k] = pme[1][k]
    opt.include_direct = int(include_direct)
    opt.include_reciprocal = int(include_reciprocal)
    b = None if box is None else _f64(box, (9,))
    f = np.zeros((n, 3))
    en = C.c_double()
    w = np.zeros(9)
    rc = lib().orc_nonbonded(n, _d(pos), _d(q), _d(s), _d(e), len(ex), _i(ei), _i(ej), _d(eqq),
                             _d(es), _d(ee), C.byref(opt), _d(b), _d(f), C.byref(en), _d(w),
                             int(threads))
    if rc != 0:
        raise ValueError(f"oracle nonbonded rejected input (code {rc})")
    if virial:
        return f, en.value, w.reshape(3, 3)
    return f, en.value


def dispersion_coefficient(sigma, epsilon, cutoff, use_switching=False, switching_distance=-1.0):
    s, e = _f64(sigma), _f64(epsilon)
    return lib().orc_dispersion_coefficient(len(s), _d(s), _d(e), cutoff, int(use_switching),
                                            switching_distance)


def pme_reciprocal(pos, charge, box, alpha, dims, virial=False):
    """PmeCache::evaluate (pme.rs:31-61, 305-425) -> (forces, energy[, virial])."""
    pos = _f64(pos, (-1, 3))
    q = _f64(charge)
    f = np.zeros_like(pos)
    w = np.zeros(9)
    d = (C.c_int * 3)(*dims)
    e = lib().orc_pme_reciprocal(pos.shape[0], _d(pos), _d(q), _d(_f64(box, (9,))),
                                 C.c_double(alpha), d, _d(f), _d(w) if virial else None)
    return (f, e, w.reshape(3, 3)) if virial else (f, e)


def ewald_reciprocal(pos, charge, box, alpha, kmax):
    pos = _f64(pos, (-1, 3))
    q = _f64(charge)
    f = np.zeros_like(pos)
    e = lib().orc_ewald_reciprocal(pos.shape[0], _d(pos), _d(q), _d(_f64(box, (9,))),
                                   C.c_double(alpha), int(kmax), _d(f))
    return f, e


def pair_set(pos, cutoff, box=None, exclusions=(), use_cells=True, max_pairs=None):
    """The reference's interacting pair set (neighbors.rs:96-181, nonbonded.rs:842-864)."""
    pos = _f64(pos, (-1, 3))
    n = pos.shape[0]
    ex = list(exclusions)
    ei = _i32([x[0] for x in ex]) if ex else np.zeros(1, np.int32)
    ej = _i32([x[1] for x in ex]) if ex else np.zeros(1, np.int32)
    b = None if box is None else _f64(box, (9,))
    count = lib().orc_pair_set(n, _d(pos), cutoff, _d(b), int(box is not None), len(ex), _i(ei),
                               _i(ej), int(use_cells), 0, None)
    out = np.zeros((max(count, 1), 2), np.int32)
    lib().orc_pair_set(n, _d(pos), cutoff, _d(b), int(box is not None), len(ex), _i(ei), _i(ej),
                       int(use_cells), count, out.ctypes.data_as(C.POINTER(C.c_int32)))
    return out[:count]


def gbsa_obc(pos, charge, radius, scale, method=0, cutoff=1.0, solvent_dielectric=78.3,
             solute_dielectric=1.0, surface_area_energy=2.25936, box=None, virial=False):
    """GBSAOBCForce::evaluate (gbsa_obc.rs:184-275) -> (forces, energy, born[, virial])."""
    pos = _f64(pos, (-1, 3))
    n = pos.shape[0]
    f = np.zeros_like(pos)
    born = np.zeros(n)
    w = np.zeros(9)
    en = C.c_double()
    b = None if box is None else _f64(box, (9,))
    rc = lib().orc_gbsa_obc(n, _d(pos), _d(_f64(charge)), _d(_f64(radius)), _d(_f64(scale)),
                            int(method), C.c_double(cutoff), C.c_double(solvent_dielectric),
                            C.c_double(solute_dielectric), C.c_double(surface_area_energy), _d(b),
                            _d(f), C.byref(en), _d(born), _d(w))
    if rc != 0:
        raise ValueError(f"oracle GBSA rejected input (code {rc})")
    return (f, en.value, born, w.reshape(3, 3)) if virial else (f, en.value, born)


def harmonic_bonds(pos, bonds, use_pbc=False, box=None, virial=False):
    """bonds: (i, j, length, k); harmonic_bond.rs:102-144."""
    pos = _f64(pos, (-1, 3))
    f = np.zeros_like(pos)
    w = np.zeros(9)
    if not bonds:
        return (f, 0.0, w.reshape(3, 3)) if virial else (f, 0.0)
    b = list(bonds)
    e = lib().orc_harmonic_bond(len(b), _i(_i32([x[0] for x in b])), _i(_i32([x[1] for x in b])),
                                _d(_f64([x[2] for x in b])), _d(_f64([x[3] for x in b])), _d(pos),
                                int(use_pbc), _d(None if box is None else _f64(box, (9,))), _d(f),
                                _d(w))
    return (f, e, w.reshape(3, 3)) if virial else (f, e)


def harmonic_angles(pos, angles, use_pbc=False, box=None, virial=False):
    """angles: (i, j, k, theta0, k_theta); harmonic_angle.rs:102-175."""
    pos = _f64(pos, (-1, 3))
    f = np.zeros_like(pos)
    w = np.zeros(9)
    if not angles:
        return (f, 0.0, w.reshape(3, 3)) if virial else (f, 0.0)
    a = list(angles)
    e = lib().orc_harmonic_angle(len(a), _i(_i32([x[0] for x in a])), _i(_i32([x[1] for x in a])),
                                 _i(_i32([x[2] for x in a])), _d(_f64([x[3] for x in a])),
                                 _d(_f64([x[4] for x in a])), _d(pos), int(use_pbc),
                                 _d(None if box is None else _f64(box, (9,))), _d(f), _d(w))
    return (f, e, w.reshape(3, 3)) if virial else (f, e)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return tuple(o)


def gaussian_noise(seed, stream, step, n):
    out = np.zeros((n, 3))
    lib().orc_gaussian_noise(seed, stream, step, n, _d(out))
    return out


def constraints_solve(constraints, masses, reference, values, velocities, tolerance):
    """ConstraintSolver::solve (constraints.rs:81-156); returns (code, values)."""
    cs = list(constraints)
    values = _f64(values, (-1, 3)).copy()
    rc = lib().orc_constraints_solve(len(cs), _i(_i32([c[0] for c in cs])),
                                     _i(_i32([c[1] for c in cs])), _d(_f64([c[2] for c in cs])),
                                     _d(_f64(masses)), _d(_f64(reference, (-1, 3))), _d(values),
                                     int(velocities), C.c_double(tolerance))
    return rc, values


def settle_positions(waters, d_oh, d_hh, masses, reference, positions):
    w = _i32(waters).reshape(-1)
    x = _f64(positions, (-1, 3)).copy()
    rc = lib().orc_settle_positions(len(w) // 3, _i(w), d_oh, d_hh, _d(_f64(masses)),
                                    _d(_f64(reference, (-1, 3))), _d(x))
    return rc, x


def settle_velocities(waters, masses, positions, velocities):
    w = _i32(waters).reshape(-1)
    v = _f64(velocities, (-1, 3)).copy()
    rc = lib().orc_settle_velocities(len(w) // 3, _i(w), _d(_f64(masses)),
                                     _d(_f64(positions, (-1, 3))), _d(v))
    return rc, v


def lfmiddle_step(pos, vel, forces, masses, dt, temperature, friction, noise, constraints=(),
                  tolerance=1e-5, mode=0, waters=None, d_oh=0.0, d_hh=0.0):
    """LangevinMiddleIntegrator::step_constrained (langevin.rs:216-278) with given normals.

    mode 0 uses the reference SHAKE/RATTLE, mode 1 analytic SETTLE for `waters`."""
    pos = _f64(pos, (-1, 3)).copy()
    vel = _f64(vel, (-1, 3)).copy()
    cs = list(constraints)
    ci = _i32([c[0] for c in cs]) if cs else np.zeros(1, np.int32)
    cj = _i32([c[1] for c in cs]) if cs else np.zeros(1, np.int32)
    cd = _f64([c[2] for c in cs]) if cs else np.zeros(1)
    w = _i32(waters).reshape(-1) if waters is not None else np.zeros(3, np.int32)
    nw = len(w) // 3 if waters is not None else 0
    rc = lib().orc_lfmiddle_step(pos.shape[0], _d(pos), _d(vel), _d(_f64(forces, (-1, 3))),
                                 _d(_f64(masses)), dt, temperature, friction,
                                 _d(_f64(noise, (-1, 3))), len(cs), _i(ci), _i(cj), _d(cd),
                                 tolerance, int(mode), nw, _i(w), d_oh, d_hh)
    return rc, pos, vel


def kinetic_energy(vel, masses):
    v = _f64(vel, (-1, 3))
    return lib().orc_kinetic_energy(v.shape[0], _d(v), _d(_f64(masses)))


def wtime():
    return lib().orc_wtime()


def max_threads():
    return lib().orc_max_threads()
