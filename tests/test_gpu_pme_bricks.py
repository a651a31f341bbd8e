"""Brick-owned PME gather against the eight-lanes-per-particle gather.

The brick form gives each CTA one brick of grid points, reads the brick and its halo of the
potential grid into shared memory and gathers the particles whose stencil starts in it; the
other form gathers each particle with eight lanes from L2.  Both sum each particle's stencil
planes in the same order, so the forces, the energy and whole trajectories must be
bit-identical between the two, and equal the oracle's (pme.rs:141-425) within the usual
tolerance.  Cases: the 23,958-atom cube (56^3 grid: four bricks per axis) and a rectangular,
non-cubic box whose grid leaves shorter bricks at the high end of every axis.
"""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems


pytestmark = pytest.mark.gpu


def stretched_box():
    """648 waters in a 2.9 x 3.4 x 4.1 nm box (each molecule moved rigidly with its oxygen)."""
    w = synth.water_box(n_waters=648, box_length=2.7, lattice=(9, 9, 8), seed=5)
    scale = np.array([2.9, 3.4, 4.1]) / 2.7
    pos = w.positions.reshape(-1, 3, 3)
    o = pos[:, :1, :]
    pos = (pos - o) + o * scale
    w.positions = pos.reshape(-1, 3)
    w.box = np.diag([2.9, 3.4, 4.1])
    return w


def water(name):
    return stretched_box() if name == "stretched" else synth.water_preset(name)


def context(w, precision, bricks, seed=7):
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(seed=seed),
                          precision=precision, pme_bricks=bricks)
    ctx.set_positions(w.positions)
    return ctx


@pytest.mark.parametrize("precision", ["mixed", "double"])
@pytest.mark.parametrize("name", ["water-23958", "stretched"])
def test_brick_forces_equal_atomic_forces(name, precision):
    w = water(name)
    on, off = context(w, precision, 1), context(w, precision, 0)
    assert on.pme_layout()["bricks_in_use"] and not off.pme_layout()["bricks_in_use"]
    a = on.get_state(forces=True, energy=True)
    b = off.get_state(forces=True, energy=True)
    assert np.array_equal(a.forces, b.forces)
    assert a.potential_energy == b.potential_energy
    f_ref, e_ref = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                               method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                               threads=8)
    err = float(np.sqrt(((a.forces - f_ref) ** 2).sum() / (f_ref ** 2).sum()))
    assert err < (5e-6 if precision == "mixed" else 1e-9)
    on.close()
    off.close()


def test_brick_trajectory_equals_atomic_trajectory():
    w = synth.water_preset("water-23958")
    on, off = context(w, "mixed", 1, seed=3), context(w, "mixed", 0, seed=3)
    for c in (on, off):
        c.set_velocities_to_temperature(300.0, seed=9)
        c.step(60)  # graph-captured groups, neighbour-list rebuilds and prunes
    a = on.get_state(positions=True, velocities=True)
    b = off.get_state(positions=True, velocities=True)
    assert on.nlist_stats()["rebuilds"] >= 2
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    on.close()
    off.close()


def nonbonded_copy(w, charges):
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method("PME")
    nb.set_cutoff_distance(0.9)
    nb.set_ewald_error_tolerance(5e-4)
    for q, s, e in zip(charges, w.sigmas(), w.epsilons()):
        nb.add_particle(float(q), float(s), float(e))
    for i, j, qq, s, e in w.exceptions():
        nb.add_exception(i, j, qq, s, e)
    return nb


def test_parameter_updates_keep_the_forms_equal():
    """A live parameter update (new charges, one of 20 e) reaches both gather forms alike."""
    w = synth.water_preset("water-1944")
    big = w.charges().copy()
    big[0], big[1] = 20.0, -19.0
    got = []
    for bricks in (1, 0):
        ctx = context(w, "mixed", bricks)
        assert ctx.pme_layout()["bricks_in_use"] == bool(bricks)
        ctx.update_nonbonded_parameters(nonbonded_copy(w, big))
        got.append(ctx.get_state(forces=True, energy=True))
        ctx.close()
    assert np.array_equal(got[0].forces, got[1].forces)
    assert got[0].potential_energy == got[1].potential_energy
