"""GBSAOBCForce on the GPU against the f64 oracle (forces/gbsa_obc.rs:184-309), through the
C ABI.  FP64 form: 1e-9 force RMS; mixed FP32 / fixed-point form: 5e-6 force RMS."""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu

K = 138.93545764438198


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def gb_context(pos, q, r, s, method=0, cutoff=1.0, solvent=78.3, solute=1.0, surface=2.25936,
               box=None, precision="double"):
    sysm = ommb200.System()
    gb = ommb200.GBSAOBCForce()
    gb.set_nonbonded_method(method)
    gb.set_cutoff_distance(cutoff)
    gb.set_solvent_dielectric(solvent)
    gb.set_solute_dielectric(solute)
    gb.set_surface_area_energy(surface)
    for qi, ri, si in zip(q, r, s):
        sysm.add_particle(1.0)
        gb.add_particle(float(qi), float(ri), float(si))
    if box is not None:
        sysm.set_default_periodic_box_vectors(*np.asarray(box))
    sysm.add_force(gb)
    ctx = ommb200.Context(sysm, systems.langevin(), precision=precision)
    ctx.set_positions(pos)
    return ctx


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_isolated_particle_known_answers(known_answers, precision):
    # tests/gbsa_obc.rs:24-58
    c = known_answers["gbsa_isolated"]
    tol = c["tolerance"] if precision == "double" else 1e-6
    for case in c["cases"]:
        ctx = gb_context([case["position"]], [case["charge"]], [case["radius"]], [1.0],
                         solvent=case["solvent"], solute=case["solute"],
                         surface=case["surface"], precision=precision)
        st = ctx.get_state(forces=True, energy=True)
        assert abs(st.potential_energy - case["expected_energy"]) < tol * max(1.0, abs(case["expected_energy"]))
        assert np.all(st.forces == 0.0)


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("surface", [0.0, 2.25936])
def test_four_particle_model_with_burial(method, surface):
    # the model of tests/gbsa_obc.rs:61-112 (unequal radii, one buried particle)
    box = np.array([[2.0, 0, 0], [0.6, 2.1, 0], [-0.4, 0.3, 2.2]])
    pos = np.array([[0.1, 0.2, 0.3], [0.135, 0.225, 0.32], [0.7, 0.4, 0.5], [1.8, 0.2, 0.3]])
    q, r, s = [0.4, -0.3, 0.2, -0.5], [0.3, 0.1, 0.17, 0.13], [1.2, 0.8, 0.7, 0.9]
    f_ref, e_ref, _ = O.gbsa_obc(pos, q, r, s, method=method, cutoff=0.9,
                                 surface_area_energy=surface, box=box)
    ctx = gb_context(pos, q, r, s, method=method, cutoff=0.9, surface=surface,
                     box=box if method == 2 else None, precision="double")
    st = ctx.get_state(forces=True, energy=True)
    assert rms_rel(st.forces, f_ref) < 1e-9
    assert abs(st.potential_energy - e_ref) < 1e-9 * abs(e_ref)


@pytest.mark.parametrize("precision,bound", [("double", 1e-9), ("mixed", 5e-6)])
def test_chain_system_matches_oracle(precision, bound):
    ch = synth.chain(600, seed=5)
    ctx = ommb200.Context(systems.chain_system(ch), systems.langevin(step_size=0.001),
                          precision=precision)
    ctx.set_positions(ch.positions)
    st = ctx.get_state(forces=True, energy=True)
    n = ch.n_atoms
    excl = sorted({(i, i + 1) for i in range(n - 1)} | {(i, i + 2) for i in range(n - 2)})
    exc = [(i, j, 0.0, ch.sigma, 0.0) for i, j in excl]
    exc += [(i, i + 3, ch.charges[i] * ch.charges[i + 3], ch.sigma, ch.epsilon) for i in range(n - 3)]
    f1, e1 = O.nonbonded(ch.positions, ch.charges, [ch.sigma] * n, [ch.epsilon] * n, exc,
                         method="NoCutoff")
    f2, e2 = O.harmonic_bonds(ch.positions, ch.bonds())
    f3, e3 = O.harmonic_angles(ch.positions, ch.angles())
    f4, e4, _ = O.gbsa_obc(ch.positions, ch.charges, ch.radii, [ch.gb_scale] * n,
                           solvent_dielectric=78.5, solute_dielectric=1.0)
    f_ref = f1 + f2 + f3 + f4
    e_ref = e1 + e2 + e3 + e4
    err = rms_rel(st.forces, f_ref)
    print(f"chain {precision}: force rms rel {err:.3e}, E {st.potential_energy:.6f} vs {e_ref:.6f}")
    assert err < bound
    assert abs(st.potential_energy - e_ref) < (1e-9 if precision == "double" else 2e-6) * abs(e_ref) + 1e-6


def test_chain_dynamics_is_stable_and_deterministic():
    ch = synth.chain(400, seed=9)
    out = []
    for _ in range(2):
        ctx = ommb200.Context(systems.chain_system(ch), systems.langevin(step_size=0.001, seed=4),
                              precision="mixed")
        ctx.set_positions(ch.positions)
        ctx.set_velocities_to_temperature(300.0, seed=2)
        ctx.step(200)
        st = ctx.get_state(positions=True, energy=True)
        assert np.isfinite(st.positions).all() and np.isfinite(st.potential_energy)
        out.append(st.positions)
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-6), ("double", 1e-10)])
def test_fused_nonbonded_gb_pass_matches_the_separate_kernels(precision, tol):
    # With the NonbondedForce and the GBSAOBCForce in different force groups, evaluating one
    # group at a time runs the nonbonded pair kernel and GB pass 2 separately; evaluating both
    # runs the nonbonded pair terms inside GB pass 2.  Both must give the same forces and the
    # same per-system energies (a batch of two chains routes energies by segment).
    chs = [synth.chain(500, seed=31), synth.chain(300, seed=32)]
    ctx = ommb200.BatchContext([systems.chain_system(c, gb_force_group=1) for c in chs],
                               systems.langevin(step_size=0.001), precision=precision)
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    both = ctx.get_state(forces=True, energy=True)
    g0 = ctx.get_state(forces=True, energy=True, groups=1 << 0)
    g1 = ctx.get_state(forces=True, energy=True, groups=1 << 1)
    split = g0.forces + g1.forces
    assert np.abs(both.forces - split).max() < tol * np.abs(split).max()
    assert abs(both.potential_energy - g0.potential_energy - g1.potential_energy) < \
        tol * abs(both.potential_energy) + 1e-6
    e_both = np.asarray(ctx.system_energies()[0])
    e_split = np.asarray(ctx.system_energies(1 << 0)[0]) + np.asarray(ctx.system_energies(1 << 1)[0])
    assert np.abs(e_both - e_split).max() < tol * np.abs(e_both).max() + 1e-6
