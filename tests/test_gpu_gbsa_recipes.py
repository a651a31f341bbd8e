"""The reference's GBSAOBCForce scenarios (tests/reference/gbsa_obc.cpp:25-72), run through the
engine and compared with the f64 oracle on the same inputs, in both precisions.

The grid: methods NoCutoff, CutoffNonPeriodic and CutoffPeriodic (cutoff 0.8 nm, a triclinic
box); 1, 2 (the second particle buried inside the first), 8 and 125 particles with the
recipe's charges, radii, scale factors and masses (the last of more than two particles is
massless); default settings, changed dielectrics and surface energy, no surface term, and a zero
solvent dielectric.  Each scenario then goes through the recipe's phases:
  0  forces and energy at the start;
  1  new per-particle parameters taken by the Context (the reference's update copies the particle
     parameters only, gbsa_obc.rs:134-141, so the dielectrics, surface energy, cutoff and method
     stay as created);
  2  a changed triclinic box and displaced positions, some shifted by a box vector;
  3  five steps of dynamics from the recipe's velocities (its Verlet integrator equals
     LangevinMiddle at zero friction and temperature), positions and velocities compared.
The reference took its expected values from an OpenMM build that is not available here, so
these cases pin the engine to the oracle's restatement of gbsa_obc.rs, not to absolute numbers.
The recipe's CustomCVForce and CustomExternalForce parts are outside the engine and left out.
"""
import math

import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import systems

pytestmark = pytest.mark.gpu

CUTOFF = 0.8
BOX0 = np.array([[3.0, 0, 0], [0.7, 3.2, 0], [-0.6, 0.4, 3.4]])
BOX2 = np.array([[3.4, 0, 0], [-0.4, 3.1, 0], [0.8, -0.6, 3.8]])
SETTINGS = [dict(solute=1.0, solvent=78.3, surface=2.25936),
            dict(solute=2.1, solvent=35.0, surface=0.75),
            dict(solute=1.0, solvent=78.3, surface=0.0),
            dict(solute=1.0, solvent=0.0, surface=2.25936)]
DT, STEPS = 0.0001, 5
# force RMS (relative, plus an absolute floor), energy (relative), position (absolute).  Forces
# accumulate in 2^-32 kJ/mol/nm fixed point, so the FP64 form carries ~1e-10 kJ/mol/nm of
# rounding, visible on the buried pair's 1e-5 kJ/mol/nm forces; the FP32 form's SFU reciprocals
# and logarithm give that pair (a 0.1 nm particle 0.05 nm inside a 0.3 nm one) about 1e-5.
BOUNDS = {"double": (1e-9, 1e-9, 1e-12), "mixed": (3e-5, 1e-5, 1e-9)}
FORCE_FLOOR = 1e-8  # kJ/mol/nm


def recipe(geometry):
    n = [1, 2, 8, 125][geometry]
    mass = np.array([0.0 if (i == n - 1 and n > 2) else 2.0 + i % 4 for i in range(n)])
    q = np.array([0.1 * (i % 7 - 3) for i in range(n)])
    r = np.array([0.11 + 0.02 * (i % 5) for i in range(n)])
    s = np.array([0.65 + 0.1 * (i % 4) for i in range(n)])
    if geometry == 1:
        r = np.array([0.3, 0.1])
        s = np.array([1.2, 1.2])
    pos = np.array([[0.37 * (i % 5) + 0.01 * math.sin(i), 0.41 * ((i // 5) % 5) + 0.02 * math.cos(i),
                     0.43 * (i // 25) + 0.015 * math.sin(2 * i)] for i in range(n)])
    if geometry == 1:
        pos[1] = pos[0] + np.array([0.035, 0.025, 0.02])
    return mass, q, r, s, pos


def oracle_forces(pos, q, r, s, method, st, box):
    f, e, _ = O.gbsa_obc(pos, q, r, s, method=method, cutoff=CUTOFF,
                         solvent_dielectric=st["solvent"], solute_dielectric=st["solute"],
                         surface_area_energy=st["surface"], box=box if method == 2 else None)
    return f, e


def compare(f, e, f_ref, e_ref, bounds):
    fb, eb, _ = bounds
    rms_ref = float(np.sqrt((f_ref ** 2).mean()))
    rms_err = float(np.sqrt(((f - f_ref) ** 2).mean()))
    assert rms_err < fb * rms_ref + FORCE_FLOOR, (rms_err, rms_ref)
    assert abs(e - e_ref) < eb * abs(e_ref) + 1e-7, (e, e_ref)


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("settings", range(4))
@pytest.mark.parametrize("geometry", range(4))
@pytest.mark.parametrize("method", range(3))
def test_reference_gbsa_scenario_matches_oracle(method, geometry, settings, precision):
    bounds = BOUNDS[precision]
    st = SETTINGS[settings]
    mass, q, r, s, pos = recipe(geometry)
    n = len(q)
    sysm = ommb200.System()
    sysm.set_default_periodic_box_vectors(*BOX0)
    gb = ommb200.GBSAOBCForce()
    gb.set_nonbonded_method(method)
    gb.set_cutoff_distance(CUTOFF)
    gb.set_solute_dielectric(st["solute"])
    gb.set_solvent_dielectric(st["solvent"])
    gb.set_surface_area_energy(st["surface"])
    for i in range(n):
        sysm.add_particle(float(mass[i]))
        gb.add_particle(float(q[i]), float(r[i]), float(s[i]))
    sysm.add_force(gb)
    ctx = ommb200.Context(sysm, systems.langevin(temperature=0.0, friction=0.0, step_size=DT),
                          precision=precision)
    ctx.set_positions(pos)
    vel = np.tile([0.01, -0.02, 0.03], (n, 1))
    ctx.set_velocities(vel)
    box = BOX0

    # phase 0: the initial state
    state = ctx.get_state(forces=True, energy=True)
    compare(state.forces, state.potential_energy, *oracle_forces(pos, q, r, s, method, st, box),
            bounds)

    # phase 1: new particle parameters (the globals stay as created)
    q, r, s = q * 0.8, r + 0.013, s * 0.97
    for i in range(n):
        gb.set_particle_parameters(i, float(q[i]), float(r[i]), float(s[i]))
    ctx.update_gbsa_obc_parameters(gb)
    state = ctx.get_state(forces=True, energy=True)
    compare(state.forces, state.potential_energy, *oracle_forces(pos, q, r, s, method, st, box),
            bounds)

    # phase 2: a new box and displaced, partly wrapped positions
    box = BOX2
    ctx.set_periodic_box_vectors(*box)
    pos = pos.copy()
    for i in range(n):
        pos[i] += [0.02 * math.sin(i + 1), -0.01 * math.cos(i), 0.015 * math.sin(i + 2)]
        if i % 3 == 1:
            pos[i] += box[1]
    ctx.set_positions(pos)
    state = ctx.get_state(forces=True, energy=True)
    compare(state.forces, state.potential_energy, *oracle_forces(pos, q, r, s, method, st, box),
            bounds)

    # phase 3: five steps at zero friction and temperature from the recipe's velocities
    ctx.step(STEPS)
    state = ctx.get_state(positions=True, velocities=True, forces=True, energy=True)
    x, v = pos.copy(), vel.copy()
    noise = np.zeros((n, 3))
    for _ in range(STEPS):
        f, _ = oracle_forces(x, q, r, s, method, st, box)
        rc, x, v = O.lfmiddle_step(x, v, f, mass, DT, 0.0, 0.0, noise)
        assert rc == 0
    assert np.abs(state.positions - x).max() < bounds[2]
    assert np.abs(state.velocities - v).max() < bounds[2] / DT
    compare(state.forces, state.potential_energy, *oracle_forces(x, q, r, s, method, st, box),
            bounds)
    ctx.close()
