"""Assemble engine Systems for the benchmark workloads from `synth` inputs."""
from __future__ import annotations

import numpy as np

from . import GBSAOBCForce, HarmonicAngleForce, HarmonicBondForce, LangevinMiddleIntegrator, NonbondedForce, System
from .synth import D_HH, D_OH, WaterBox


def water_system(w: WaterBox, cutoff: float = 0.9, ewald_tolerance: float = 5e-4,
                 method: str = "PME", dispersion_correction: bool = True,
                 switching_distance: float | None = None, constraints: bool = True) -> System:
    """Rigid 3-site water: NonbondedForce (PME by default) with 3 exclusions per molecule and
    O-H / O-H / H-H distance constraints (solved by SETTLE in the engine)."""
    system = System()
    for m in w.masses():
        system.add_particle(float(m))
    b = w.box
    system.set_default_periodic_box_vectors(b[0], b[1], b[2])
    nb = NonbondedForce()
    nb.set_nonbonded_method(method)
    nb.set_cutoff_distance(cutoff)
    nb.set_ewald_error_tolerance(ewald_tolerance)
    nb.set_use_dispersion_correction(dispersion_correction)
    if switching_distance is not None:
        nb.set_use_switching_function(True)
        nb.set_switching_distance(switching_distance)
    for q, s, e in zip(w.charges(), w.sigmas(), w.epsilons()):
        nb.add_particle(float(q), float(s), float(e))
    for i, j, qq, s, e in w.exceptions():
        nb.add_exception(i, j, qq, s, e)
    system.add_force(nb)
    if constraints:
        for i, j, d in w.constraints():
            system.add_constraint(i, j, d)
    return system


def langevin(temperature=300.0, friction=1.0, step_size=0.002, seed=1234):
    integ = LangevinMiddleIntegrator(temperature, friction, step_size)
    integ.set_random_number_seed(seed)
    return integ


def chain_system(chain, coulomb14=1.0, lj14=1.0, gbsa=True, solvent_dielectric=78.5,
                 solute_dielectric=1.0, surface_area_energy=2.25936, cutoff=None,
                 learned_radii=None, gb_force_group=0) -> System:
    """One implicit-solvent chain: NonbondedForce with 1-2/1-3 exclusions and 1-4 exceptions,
    harmonic bonds and angles, and (by default) a GBSAOBCForce; NoCutoff, or
    CutoffNonPeriodic for both forces when `cutoff` (nm) is given.  `learned_radii`: keyword
    arguments of GBSAOBCForce.set_learned_radii (None = exact OBC)."""
    system = System()
    for _ in range(chain.n_atoms):
        system.add_particle(chain.mass)
    nb = NonbondedForce()
    if cutoff is None:
        nb.set_nonbonded_method("NoCutoff")
    else:
        nb.set_nonbonded_method("CutoffNonPeriodic")
        nb.set_cutoff_distance(cutoff)
    for q in chain.charges:
        nb.add_particle(float(q), chain.sigma, chain.epsilon)
    bonds = [(i, i + 1) for i in range(chain.n_atoms - 1)]
    nb.create_exceptions_from_bonds(bonds, coulomb14, lj14)
    system.add_force(nb)
    hb = HarmonicBondForce()
    for i, j, r0, k in chain.bonds():
        hb.add_bond(i, j, r0, k)
    system.add_force(hb)
    ha = HarmonicAngleForce()
    for i, j, k, th, kt in chain.angles():
        ha.add_angle(i, j, k, th, kt)
    system.add_force(ha)
    if gbsa:
        gb = GBSAOBCForce()
        if cutoff is not None:
            gb.set_nonbonded_method(1)
            gb.set_cutoff_distance(cutoff)
        gb.set_solvent_dielectric(solvent_dielectric)
        gb.set_solute_dielectric(solute_dielectric)
        gb.set_surface_area_energy(surface_area_energy)
        for q, r in zip(chain.charges, chain.radii):
            gb.add_particle(float(q), float(r), chain.gb_scale)
        if learned_radii is not None:
            gb.set_learned_radii(**learned_radii)
        gb.set_force_group(gb_force_group)
        system.add_force(gb)
    return system


__all__ = ["water_system", "chain_system", "langevin", "D_OH", "D_HH", "np"]
