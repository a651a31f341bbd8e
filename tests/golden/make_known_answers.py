"""Generates tests/golden/known_answers.json: the reference's analytic known-answer cases.

The reference (mogura-rs/openmm-rs) commits no golden output vectors for this path; its
OpenMM-generated fixtures need an external OpenMM checkout.  What it does commit are analytic
known-answer tests.  This script restates their inputs and closed-form expected values (no
oracle or engine output is written here), citing the test each case comes from:

* nonbonded.rs:1457-1472  test_coulomb
* nonbonded.rs:1474-1494  test_lj
* nonbonded.rs:1497-1515  test_exclusions
* tests/gbsa_obc.rs:24-58 isolated_gbsa_matches_born_and_surface_energies
* tests/integrator_compatibility.rs:38-58 langevin_middle_matches_reference_zero_temperature_update
* harmonic_bond.rs:187-228  test_bonds, test_periodic
* harmonic_angle.rs:212-259 test_equilibrium, test_displaced_angle, test_conservation
* Random123 kat_vectors for philox4x32_10 (Salmon et al., SC'11)

Run:  python tests/golden/make_known_answers.py
"""
import json
import math
from pathlib import Path

ONE_4PI_EPS0 = 138.93545764438198


def main():
    cases = {}
    # nonbonded.rs:1457-1472
    cases["coulomb"] = dict(
        positions=[[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]], charge=[0.5, -1.5], sigma=[1.0, 1.0],
        epsilon=[0.0, 0.0], exceptions=[], method="NoCutoff",
        expected_force0_x=-ONE_4PI_EPS0 * (-0.75) / 4.0,
        expected_force1_x=ONE_4PI_EPS0 * (-0.75) / 4.0,
        expected_energy=ONE_4PI_EPS0 * (-0.75) / 2.0, tolerance=1e-4)
    # nonbonded.rs:1474-1494
    sigma, eps = 1.3, math.sqrt(2.0)
    x = sigma / 2.0
    cases["lj"] = dict(
        positions=[[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]], charge=[0.0, 0.0], sigma=[1.2, 1.4],
        epsilon=[1.0, 2.0], exceptions=[], method="NoCutoff",
        expected_energy=4.0 * eps * (x ** 12 - x ** 6),
        expected_force0_x=4.0 * eps * (-12.0 * x ** 12 + 6.0 * x ** 6) / 2.0,
        expected_force1_x=-4.0 * eps * (-12.0 * x ** 12 + 6.0 * x ** 6) / 2.0, tolerance=1e-4)
    # nonbonded.rs:1497-1515
    cases["exclusions"] = dict(
        positions=[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [2.0, 0.0, 0.0]], charge=[1.0, 1.0, 1.0],
        sigma=[1.0, 1.0, 1.0], epsilon=[1.0, 1.0, 1.0],
        exceptions=[[0, 1, 0.0, 1.0, 0.0], [0, 2, 0.0, 1.0, 0.0]], method="NoCutoff",
        expected_force0=[0.0, 0.0, 0.0], tolerance=1e-5)
    # tests/gbsa_obc.rs:24-58
    iso = []
    for solute, solvent, surface in [(1.0, 78.3, 2.25936), (2.1, 35.0, 0.75), (0.0, 78.3, 2.25936),
                                     (1.0, 0.0, 0.0)]:
        for radius in [0.005, 0.008, 0.15]:
            born = radius - 0.009
            elec = 0.0 if solute == 0.0 or solvent == 0.0 else (
                -0.5 * ONE_4PI_EPS0 * 0.25 * (1.0 / solute - 1.0 / solvent) / abs(born))
            area = (4.0 * math.pi * surface * (radius + 0.14) ** 2 * (radius / born) ** 6
                    if born > 0.0 else 0.0)
            iso.append(dict(solute=solute, solvent=solvent, surface=surface, radius=radius,
                            charge=0.5, position=[0.2, 0.3, 0.4], expected_energy=elec + area))
    cases["gbsa_isolated"] = dict(cases=iso, tolerance=1e-10)
    # tests/integrator_compatibility.rs:38-58
    v = 0.5 * math.exp(-0.2)
    cases["lfmiddle_zero_temperature"] = dict(
        temperature=0.0, friction=2.0, step_size=0.1, position=[1.0, 0.0, 0.0],
        velocity=[0.3, 0.0, 0.0], force=[4.0, 0.0, 0.0], mass=2.0, expected_velocity_x=v,
        expected_position_x=1.0 + 0.05 * (0.5 + v), tolerance=2e-7)
    # harmonic_bond.rs:187-208: bonds (0, 1, 1.5, 0.8) and (1, 2, 1.2, 0.7) (i, j, length, k)
    cases["harmonic_bonds"] = dict(
        positions=[[0.0, 2.0, 0.0], [0.0, 0.0, 0.0], [1.0, 0.0, 0.0]],
        bonds=[[0, 1, 1.5, 0.8], [1, 2, 1.2, 0.7]],
        expected_force0_y=-0.8 * 0.5, expected_force2_x=0.7 * 0.2,
        expected_energy=0.5 * 0.8 * 0.25 + 0.5 * 0.7 * 0.04, tolerance=1e-5)
    # harmonic_bond.rs:210-228: the minimum image across a 3 nm cubic box
    cases["harmonic_bond_periodic"] = dict(
        positions=[[0.0, 2.0, 0.0], [0.0, 0.0, 0.0]], bonds=[[0, 1, 1.2, 0.8]],
        box=[[3.0, 0.0, 0.0], [0.0, 3.0, 0.0], [0.0, 0.0, 3.0]],
        expected_energy=0.5 * 0.8 * 0.04, tolerance=1e-5)
    # harmonic_angle.rs:212-259 (i, j, k, theta0, k_theta)
    cases["harmonic_angles"] = dict(
        equilibrium=dict(positions=[[1.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0]],
                         angles=[[0, 1, 2, math.pi / 2, 1.0]], expected_energy=0.0,
                         energy_tolerance=1e-5, force_tolerance=1e-4),
        displaced=dict(positions=[[1.0, 0.0, 0.0], [0.0, 0.0, 0.0], [1.0, 1.0, 0.0]],
                       angles=[[0, 1, 2, math.pi / 2, 2.0]],
                       expected_energy=0.5 * 2.0 * (math.pi / 4 - math.pi / 2) ** 2,
                       energy_tolerance=1e-5),
        conservation=dict(positions=[[1.2, 0.3, 0.0], [0.0, 0.0, 0.0], [0.4, 1.1, 0.0]],
                          angles=[[0, 1, 2, math.pi / 2, 1.5]], force_sum_tolerance=1e-4))
    # Random123 philox4x32_10 known-answer vectors
    cases["philox4x32_10"] = [
        dict(ctr=[0, 0, 0, 0], key=[0, 0],
             out=[0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        dict(ctr=[0xFFFFFFFF] * 4, key=[0xFFFFFFFF] * 2,
             out=[0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        dict(ctr=[0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], key=[0xA4093822, 0x299F31D0],
             out=[0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    out = Path(__file__).with_name("known_answers.json")
    out.write_text(json.dumps(cases, indent=1) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
