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


# ---- learned Born radii (no reference counterpart; OBC terms from gbsa_obc.rs:184-309) ----
# Feature and switch constants; the engine's learned-radii path uses the same values.
LR_NF = 32                       # radial symmetry functions per particle
LR_MU0, LR_DMU = 0.1, 1.1 / 31   # Gaussian centres 0.1 .. 1.2 nm
LR_ETA = 1.0 / (2.0 * 0.07 ** 2)  # Gaussian width 0.07 nm
LR_RF = 1.2                      # feature cutoff (nm)
LR_RC, LR_RS = 2.0, 1.8          # short-range integral cutoff and switch start (nm)
LR_HIDDEN = 64
# flat float32 parameter block: W1[32][64], b1[64], W2[64][64], b2[64], w3[64], b3, then the
# fixed normalisation: feature mean[32], feature 1/std[32], target mean, target scale
LR_OFF = {"W1": 0, "b1": 2048, "W2": 2112, "b2": 6208, "w3": 6272, "b3": 6336, "mean": 6337,
          "inv_std": 6369, "t_mean": 6401, "t_scale": 6402}
LR_N_PARAMS = 6403
LR_N_TRAIN = 6337


def radial_features(pos, nf=LR_NF, mu0=LR_MU0, dmu=LR_DMU, eta=LR_ETA, rc=LR_RF):
    """Radial symmetry functions (Behler & Parrinello 2007) G [n][nf] in f64."""
    pos = _f64(pos, (-1, 3))
    n = pos.shape[0]
    g = np.zeros((n, nf))
    rcode = lib().orc_radial_features(n, _d(pos), nf, C.c_double(mu0), C.c_double(dmu),
                                      C.c_double(eta), C.c_double(rc), _d(g))
    if rcode != 0:
        raise ValueError("oracle rejected feature parameters")
    return g


def learned_gbsa(pos, charge, radius, scale, tail, dtail_dg, solvent_dielectric=78.5,
                 solute_dielectric=1.0, surface_area_energy=2.25936, rs=LR_RS, rc=LR_RC,
                 rf=LR_RF, nf=LR_NF, mu0=LR_MU0, dmu=LR_DMU, eta=LR_ETA):
    """GB energy/forces with I = I_short + tail -> (forces, energy, born, I_short, I_full)."""
    pos = _f64(pos, (-1, 3))
    n = pos.shape[0]
    f = np.zeros_like(pos)
    born, short, full = np.zeros(n), np.zeros(n), np.zeros(n)
    en = C.c_double()
    rcode = lib().orc_learned_gbsa(
        n, _d(pos), _d(_f64(charge)), _d(_f64(radius)), _d(_f64(scale)),
        C.c_double(solvent_dielectric), C.c_double(solute_dielectric),
        C.c_double(surface_area_energy), C.c_double(rs), C.c_double(rc), C.c_double(rf), nf,
        C.c_double(mu0),
        C.c_double(dmu), C.c_double(eta), _d(_f64(tail)), _d(_f64(dtail_dg, (-1,))), _d(f),
        C.byref(en), _d(born), _d(short), _d(full))
    if rcode != 0:
        raise ValueError("oracle rejected learned-GB parameters")
    return f, en.value, born, short, full


def bf16(x):
    """Round to bfloat16 (nearest even) through float32, returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    a = ((a + (((a >> 16) & 1) + 0x7FFF)) >> 16) << 16
    return a.astype(np.uint32).view(np.float32).astype(np.float64)


def mlp_unpack(params):
    p = np.asarray(params, dtype=np.float32)
    o = LR_OFF
    return {"W1": p[o["W1"]:o["b1"]].reshape(32, 64), "b1": p[o["b1"]:o["W2"]],
            "W2": p[o["W2"]:o["b2"]].reshape(64, 64), "b2": p[o["b2"]:o["w3"]],
            "w3": p[o["w3"]:o["b3"]], "b3": p[o["b3"]], "mean": p[o["mean"]:o["inv_std"]],
            "inv_std": p[o["inv_std"]:o["t_mean"]], "t_mean": p[o["t_mean"]],
            "t_scale": p[o["t_scale"]]}


def mlp_forward(params, features, quantize=True):
    """32 -> 64 -> 64 -> 1 tanh network on normalised features, with the tensor-core kernels'
    rounding points (BF16 inputs, weights and first-layer activations; wider sums in f64).
    Returns (y, cache); y is the normalised tail."""
    P = mlp_unpack(params)
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    if quantize:  # the kernels normalise in float32
        x = ((np.asarray(features, np.float32) - P["mean"]) * P["inv_std"]).astype(np.float32)
    else:
        x = (np.asarray(features, np.float64) - P["mean"]) * P["inv_std"].astype(np.float64)
    xq, w1, w2 = q(x), q(P["W1"]), q(P["W2"])
    z1 = xq @ w1 + P["b1"].astype(np.float64)
    h1 = np.tanh(z1)
    h1q = q(h1)
    z2 = h1q @ w2 + P["b2"].astype(np.float64)
    h2 = np.tanh(z2)
    y = h2 @ P["w3"].astype(np.float64) + float(P["b3"])
    return y, {"xq": xq, "w1": w1, "w2": w2, "h1": h1, "h1q": h1q, "h2": h2, "P": P, "q": q}


def mlp_input_grad(cache):
    """d y / d features [n][32] (through the normalisation), same rounding points."""
    P, q = cache["P"], cache["q"]
    d2q = q(P["w3"].astype(np.float64) * (1.0 - cache["h2"] ** 2))
    d1q = q((d2q @ cache["w2"].T) * (1.0 - cache["h1"] ** 2))
    return (d1q @ cache["w1"].T) * P["inv_std"].astype(np.float64)


def mlp_loss_grad(params, features, targets, quantize=True):
    """Mean squared error of the normalised tail over the batch and its gradient with respect
    to the trainable parameters (flat, LR_N_TRAIN), with the training kernel's rounding."""
    y, c = mlp_forward(params, features, quantize)
    P, q = c["P"], c["q"]
    t = ((np.asarray(targets, np.float32) - P["t_mean"]) / P["t_scale"]).astype(np.float64)
    b = len(y)
    g = 2.0 * (y - t) / b
    d2 = g[:, None] * P["w3"].astype(np.float64) * (1.0 - c["h2"] ** 2)
    d2q = q(d2)
    d1 = (d2q @ c["w2"].T) * (1.0 - c["h1"] ** 2)
    d1q = q(d1)
    grad = np.zeros(LR_N_TRAIN)
    o = LR_OFF
    grad[o["W1"]:o["b1"]] = (c["xq"].T @ d1q).reshape(-1)
    grad[o["b1"]:o["W2"]] = d1.sum(0)
    grad[o["W2"]:o["b2"]] = (c["h1q"].T @ d2q).reshape(-1)
    grad[o["b2"]:o["w3"]] = d2.sum(0)
    grad[o["w3"]:o["b3"]] = c["h2"].T @ g
    grad[o["b3"]] = g.sum()
    return float(np.mean((y - t) ** 2)), grad


def adam_update(params, m, v, grad, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """Adam (Kingma & Ba, ICLR 2015), step t >= 1, on the trainable block; in place."""
    k = LR_N_TRAIN
    m[:k] = beta1 * m[:k] + (1 - beta1) * grad
    v[:k] = beta2 * v[:k] + (1 - beta2) * grad * grad
    mh = m[:k] / (1 - beta1 ** t)
    vh = v[:k] / (1 - beta2 ** t)
    params[:k] = params[:k] - lr * mh / (np.sqrt(vh) + eps)
    return params, m, v


# ---- MonteCarloBarostat (forces/barostat.rs, system.rs, context.rs), pure Python ----------
BOLTZMANN = 1.380649e-23 * 6.02214076e23 / 1000.0  # kJ/mol/K (integrators/langevin.rs)
BAR_NM3_TO_KJ_PER_MOL = 0.0602214076                # barostat.rs:13


def molecules(n, constraints=(), bonds=()):
    """system.rs:100-141: particles joined by constraints and bonds (union-find whose root is
    the smaller index), each molecule's particles in increasing order, molecules ordered by
    their first particle."""
    parent = list(range(n))

    def root(p):
        while parent[p] != p:
            parent[p] = parent[parent[p]]
            p = parent[p]
        return p

    for a, b in list(constraints) + list(bonds):
        ra, rb = root(a), root(b)
        parent[max(ra, rb)] = min(ra, rb)
    groups = [[] for _ in range(n)]
    for i in range(n):
        groups[root(i)].append(i)
    return [g for g in groups if g]


def scale_positions(pos, mols, scale, rigid):
    """context.rs:976-1028 with the diagonal transform of an isotropic move: every coordinate
    times `scale`, or each molecule shifted by (scale - 1) times its unweighted centroid."""
    out = np.array(pos, dtype=np.float64).reshape(-1, 3).copy()
    if not rigid:
        return scale * out
    f = scale - 1.0
    for m in mols:
        c = np.zeros(3)
        for a in m:
            c = c + out[a]
        c = c * (1.0 / len(m))
        out[m] = out[m] + f * c
    return out


def barostat_work(energy_change, pressure, old_volume, new_volume, scaled, temperature):
    """barostat.rs:144-148"""
    kt = BOLTZMANN * temperature
    return (energy_change + pressure * BAR_NM3_TO_KJ_PER_MOL * (new_volume - old_volume)
            - scaled * kt * np.log(new_volume / old_volume))


def barostat_accepts(work, temperature, uniform):
    """barostat.rs:149-160: `uniform` is drawn only when the work is positive."""
    kt = BOLTZMANN * temperature
    if np.isnan(work):
        return False
    if work <= 0.0:
        return True
    return bool(kt > 0.0 and uniform <= np.exp(-work / kt))


class VolumeStep:
    """barostat.rs:172-189 and 202-204: the volume step starts at 1 % of the volume and adapts
    every 10 attempts."""

    def __init__(self, volume):
        self.scale, self.attempted, self.accepted = 0.01 * volume, 0, 0

    def record(self, accepted, previous_volume):
        self.attempted += 1
        self.accepted += int(accepted)
        if self.attempted >= 10:
            fraction = self.accepted / self.attempted
            if fraction < 0.25:
                self.scale /= 1.1
            elif fraction > 0.75:
                self.scale = min(self.scale * 1.1, previous_volume * 0.3)
            else:
                return
            self.attempted = self.accepted = 0
