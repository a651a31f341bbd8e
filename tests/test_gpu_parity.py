"""GPU parity of the engine against the f64 CPU oracle, through the C ABI (Python ctypes).

Tolerances: FP64 form of the kernels agrees with the oracle to 1e-9 relative (force RMS)
and 1e-9 relative (energy); the mixed FP32 / fixed-point form to the accuracy target of
5e-6 force RMS relative error.  The interacting pair set must equal the reference's exactly.
"""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu

MIXED_FORCE_RMS = 5e-6
DOUBLE_FORCE_RMS = 1e-9


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def water(name):
    return synth.water_preset(name)


def oracle_water(w, threads=8, virial=False):
    return O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                       method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                       threads=threads, virial=virial)


def make_context(w, precision, seed=7, **kw):
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(seed=seed), precision=precision,
                          **kw)
    ctx.set_positions(w.positions)
    return ctx


_ORACLE_CACHE = {}


def oracle_cached(name):
    if name not in _ORACLE_CACHE:
        _ORACLE_CACHE[name] = oracle_water(water(name), virial=True)
    return _ORACLE_CACHE[name]


# --- known answers through the engine -----------------------------------------------------
@pytest.mark.parametrize("precision", ["mixed", "double"])
@pytest.mark.parametrize("name", ["coulomb", "lj", "exclusions"])
def test_engine_known_answers(known_answers, name, precision):
    c = known_answers[name]  # nonbonded.rs:1457-1515
    s = ommb200.System()
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method(c["method"])
    for q, sg, e in zip(c["charge"], c["sigma"], c["epsilon"]):
        s.add_particle(1.0)
        nb.add_particle(q, sg, e)
    for ex in c["exceptions"]:
        nb.add_exception(*ex)
    s.add_force(nb)
    ctx = ommb200.Context(s, systems.langevin(), precision=precision)
    ctx.set_positions(c["positions"])
    st = ctx.get_state(forces=True, energy=True)
    tol = c["tolerance"]
    if "expected_energy" in c:
        assert abs(st.potential_energy - c["expected_energy"]) < tol
        assert abs(st.forces[0, 0] - c["expected_force0_x"]) < tol
        assert abs(st.forces[1, 0] - c["expected_force1_x"]) < tol
    else:
        assert np.abs(st.forces[0] - np.array(c["expected_force0"])).max() < tol


def test_engine_zero_temperature_known_answer(known_answers):
    # tests/integrator_compatibility.rs:38-58; the force of 4 kJ/mol/nm comes from a harmonic
    # bond (k = 1, r0 = 5) to a massless anchor at the origin, which the integrator never moves.
    c = known_answers["lfmiddle_zero_temperature"]
    s = ommb200.System()
    s.add_particle(c["mass"])
    s.add_particle(0.0)
    hb = ommb200.HarmonicBondForce()
    hb.add_bond(0, 1, 5.0, 1.0)
    s.add_force(hb)
    integ = ommb200.LangevinMiddleIntegrator(c["temperature"], c["friction"], c["step_size"])
    integ.set_random_number_seed(3)
    ctx = ommb200.Context(s, integ, precision="double")
    ctx.set_positions([c["position"], [0.0, 0.0, 0.0]])
    ctx.set_velocities([c["velocity"], [0.0, 0.0, 0.0]])
    ctx.step(1)
    st = ctx.get_state(positions=True, velocities=True)
    assert abs(st.velocities[0, 0] - c["expected_velocity_x"]) < c["tolerance"]
    assert abs(st.positions[0, 0] - c["expected_position_x"]) < c["tolerance"]
    assert np.all(st.positions[1] == 0.0)


# --- water boxes against the oracle ---------------------------------------------------------
@pytest.mark.parametrize("precision,bound", [("mixed", MIXED_FORCE_RMS), ("double", DOUBLE_FORCE_RMS)])
@pytest.mark.parametrize("name", ["water-1944", "water-23958"])
def test_water_forces_and_energy_match_oracle(name, precision, bound):
    w = water(name)
    f_ref, e_ref, vir_ref = oracle_cached(name)
    ctx = make_context(w, precision)
    st = ctx.get_state(forces=True, energy=True, virial=True)
    err = rms_rel(st.forces, f_ref)
    print(f"{name} {precision}: force rms rel {err:.3e} energy {st.potential_energy:.6f} vs {e_ref:.6f}")
    assert err < bound
    e_tol = 2e-6 if precision == "mixed" else 1e-9
    assert abs(st.potential_energy - e_ref) < e_tol * abs(e_ref) + 1e-6 * w.n_atoms
    v_tol = 1e-4 if precision == "mixed" else 1e-8
    assert np.abs(st.virial - vir_ref).max() < v_tol * np.abs(vir_ref).max()


@pytest.mark.parametrize("name", ["water-1944", "water-23958"])
def test_pair_set_is_the_reference_pair_set(name):
    w = water(name)
    ref = O.pair_set(w.positions, 0.9, box=w.box, exclusions=[e[:2] for e in w.exceptions()])
    for precision in ("mixed", "double"):
        ctx = make_context(w, precision)
        got = ctx.debug_pair_list()
        assert len(got) == len(ref), (precision, len(got), len(ref))
        a = np.sort(got[:, 0].astype(np.int64) * 10_000_000 + got[:, 1])
        b = np.sort(ref[:, 0].astype(np.int64) * 10_000_000 + ref[:, 1])
        assert np.array_equal(a, b), precision


def test_pair_set_after_dynamics_and_rebuilds():
    w = water("water-1944")
    ctx = make_context(w, "mixed")
    ctx.set_velocities_to_temperature(300.0, seed=5)
    ctx.step(60)
    pos = ctx.get_state(positions=True).positions
    ref = O.pair_set(pos, 0.9, box=w.box, exclusions=[e[:2] for e in w.exceptions()])
    got = ctx.debug_pair_list()
    a = np.sort(got[:, 0].astype(np.int64) * 10_000_000 + got[:, 1])
    b = np.sort(ref[:, 0].astype(np.int64) * 10_000_000 + ref[:, 1])
    assert np.array_equal(a, b)


def test_switching_and_reaction_field_match_oracle():
    w = synth.water_box(300, 2.2, (7, 7, 7), seed=11)
    for method in ("CutoffPeriodic", "PME"):
        s = systems.water_system(w, cutoff=1.0, method=method, switching_distance=0.8)
        ctx = ommb200.Context(s, systems.langevin(), precision="double")
        ctx.set_positions(w.positions)
        st = ctx.get_state(forces=True, energy=True)
        f, e = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                           method=method, cutoff=1.0, box=w.box, use_switching=True,
                           switching_distance=0.8)
        assert rms_rel(st.forces, f) < 1e-9, method
        assert abs(st.potential_energy - e) < 1e-8 * abs(e) + 1e-8, method


def test_no_cutoff_chain_matches_oracle():
    ch = synth.chain(300, seed=3)
    for precision, bound in (("double", 1e-9), ("mixed", 5e-6)):
        ctx = ommb200.Context(systems.chain_system(ch, gbsa=False),
                              systems.langevin(step_size=0.001), precision=precision)
        ctx.set_positions(ch.positions)
        st = ctx.get_state(forces=True, energy=True)
        exc = _chain_exceptions(ch)
        f1, e1 = O.nonbonded(ch.positions, ch.charges, [ch.sigma] * ch.n_atoms,
                             [ch.epsilon] * ch.n_atoms, exc, method="NoCutoff")
        f2, e2 = O.harmonic_bonds(ch.positions, ch.bonds())
        f3, e3 = O.harmonic_angles(ch.positions, ch.angles())
        f_ref = f1 + f2 + f3
        e_ref = e1 + e2 + e3
        assert rms_rel(st.forces, f_ref) < bound, precision
        assert abs(st.potential_energy - e_ref) < 1e-6 * abs(e_ref) + 1e-6, precision


def _chain_exceptions(ch):
    n = ch.n_atoms
    excl = set()
    for i in range(n - 1):
        excl.add((i, i + 1))
    for i in range(n - 2):
        excl.add((i, i + 2))
    out = [(i, j, 0.0, ch.sigma, 0.0) for (i, j) in sorted(excl)]
    for i in range(n - 3):
        out.append((i, i + 3, ch.charges[i] * ch.charges[i + 3], ch.sigma, ch.epsilon))
    return out


# --- integration ----------------------------------------------------------------------------
def test_lfmiddle_settle_step_matches_oracle():
    w = water("water-1944")
    seed = 99
    ctx = make_context(w, "double", seed=seed)
    rng = np.random.default_rng(0)
    v0 = rng.normal(scale=0.3, size=(w.n_atoms, 3))
    _, v0 = O.settle_velocities(w.waters(), w.masses(), w.positions, v0)
    ctx.set_velocities(v0)
    ctx.step(1)
    st = ctx.get_state(positions=True, velocities=True)
    f, _ = oracle_water(w)
    noise = O.gaussian_noise(seed, 0, 0, w.n_atoms)
    rc, x, v = O.lfmiddle_step(w.positions, v0, f, w.masses(), 0.002, 300.0, 1.0, noise, mode=1,
                               waters=w.waters(), d_oh=synth.D_OH, d_hh=synth.D_HH)
    assert rc == 0
    assert np.abs(st.positions - x).max() < 1e-10
    assert np.abs(st.velocities - v).max() < 1e-8


def test_rigid_water_constraints_preserved():
    # tests/constraints.rs:41-76
    s = ommb200.System()
    for m in (16.0, 1.0, 1.0):
        s.add_particle(m)
    for i, j, d in ((0, 1, 0.1), (0, 2, 0.1), (1, 2, 0.16)):
        s.add_constraint(i, j, d)
    integ = ommb200.LangevinMiddleIntegrator(300.0, 2.0, 0.001)
    integ.set_random_number_seed(17)
    ctx = ommb200.Context(s, integ, precision="double")
    ctx.set_positions([[0.0, 0.0, 0.0], [0.08, 0.06, 0.0], [-0.08, 0.06, 0.0]])
    ctx.set_velocities([[0.2, 0.1, 0.0]] * 3)
    for _ in range(100):
        ctx.step(1)
        p = ctx.get_state(positions=True).positions
        for i, j, d in ((0, 1, 0.1), (0, 2, 0.1), (1, 2, 0.16)):
            assert abs(np.linalg.norm(p[i] - p[j]) / d - 1) < 2e-5


def test_shake_cluster_preserves_center_of_mass_projection():
    # tests/constraints.rs:15-39 through apply_constraints / apply_velocity_constraints
    s = ommb200.System()
    s.add_particle(1.0)
    s.add_particle(2.0)
    s.add_constraint(0, 1, 1.0)
    ctx = ommb200.Context(s, ommb200.LangevinMiddleIntegrator(0.0, 1.0, 0.001), precision="double")
    ctx.set_positions([[0, 0, 0], [1.2, 0, 0]])
    ctx.set_velocities([[1, 2, 0], [-1, -1, 0]])
    ctx.apply_constraints(1e-6)
    ctx.apply_velocity_constraints(1e-6)
    st = ctx.get_state(positions=True, velocities=True)
    p, v = st.positions, st.velocities
    assert abs(p[1, 0] - p[0, 0] - 1.0) < 2e-6 and abs(p[0, 0] + 2 * p[1, 0] - 2.4) < 2e-6
    assert abs(v[1, 0] - v[0, 0]) < 2e-6 and abs(v[0, 0] + 2 * v[1, 0] + 1.0) < 2e-6
    assert v[0, 1] == 2.0 and v[1, 1] == -1.0


def test_singular_projection_reports_constraint_error():
    # tests/constraints.rs:77-97
    s = ommb200.System()
    s.add_particle(1.0)
    s.add_particle(1.0)
    s.add_constraint(0, 1, 1.0)
    ctx = ommb200.Context(s, ommb200.LangevinMiddleIntegrator(0.0, 1.0, 0.001), precision="double")
    ctx.set_positions(np.zeros((2, 3)))
    with pytest.raises(ommb200.ConstraintError):
        ctx.apply_constraints(1e-5)


def test_nonfinite_position_is_rejected_on_the_host():
    # neighbors.rs:107-110 asserts finite positions; the engine rejects them before any launch
    w = synth.water_box(64, 1.9, (4, 4, 4), seed=2)
    ctx = make_context(w, "mixed")
    pos = w.positions.copy()
    pos[5, 1] = np.nan
    with pytest.raises(ommb200.InvalidArgument):
        ctx.set_positions(pos)
    ctx.step(2)  # the context is still usable with its previous positions


def test_runs_are_bit_identical():
    w = water("water-1944")
    out = []
    for _ in range(2):
        ctx = make_context(w, "mixed", seed=42)
        ctx.set_velocities_to_temperature(300.0, seed=9)
        ctx.step(40)
        st = ctx.get_state(positions=True, velocities=True, forces=True)
        out.append((st.positions, st.velocities, st.forces))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_graph_and_stream_paths_agree():
    w = water("water-1944")
    res = []
    for graph in (True, False):
        ctx = make_context(w, "mixed", seed=5, use_cuda_graph=graph, steps_per_graph=10)
        ctx.set_velocities_to_temperature(300.0, seed=1)
        ctx.step(30)
        res.append(ctx.get_state(positions=True).positions)
    assert np.array_equal(res[0], res[1])


def equilibrated_water(name="water-1944", steps=3000):
    """The lattice start relaxes by ~27 MJ/mol; a strongly coupled bath (20/ps) removes that
    heat before a test measures anything."""
    w = water(name)
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(friction=20.0, seed=31),
                          precision="mixed")
    ctx.set_positions(w.positions)
    ctx.set_velocities_to_temperature(300.0, seed=4)
    ctx.step(steps)
    st = ctx.get_state(positions=True, velocities=True)
    return w, st.positions, st.velocities


def test_autotune_keeps_the_trajectory():
    w = water("water-1944")
    out = []
    for tune in (False, True):
        ctx = make_context(w, "mixed", seed=21)
        ctx.set_velocities_to_temperature(300.0, seed=6)
        if tune:
            t = ctx.autotune(40)
            assert 0.05 < t["skin_nm"] <= 0.2 and t["pair_ctas_per_sm"] in range(2, 13)
            assert t["cull_tiles"] in (0, 4, 8, 16, 32, 64)
        ctx.step(30)
        st = ctx.get_state(positions=True, velocities=True)
        out.append((st.positions, st.velocities, st.step_count))
    # the skin and the pair kernel's form change how pairs are grouped into tiles and rounds
    # (so float summation order), never which pairs interact or the random stream: the
    # trajectories agree to rounding
    assert np.abs(out[0][0] - out[1][0]).max() < 1e-6
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-3
    assert out[0][2] == out[1][2] == 30


def test_thermostat_temperature():
    w, x, v = equilibrated_water()
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(friction=5.0, seed=8),
                          precision="mixed")
    ctx.set_positions(x)
    ctx.set_velocities(v)
    ctx.step(500)
    kb = 1.380649e-23 * 6.02214076e23 / 1000.0
    dof = 6 * w.n_waters
    ke = []
    for _ in range(40):
        ctx.step(50)
        ke.append(ctx.get_state(energy=True).kinetic_energy)
    t = 2 * np.mean(ke) / (dof * kb)
    assert abs(t - 300.0) < 9.0, t


def test_force_groups_split_direct_and_reciprocal():
    w = synth.water_box(100, 2.0, (5, 5, 4), seed=4)
    s = ommb200.System()
    for m in w.masses():
        s.add_particle(float(m))
    s.set_default_periodic_box_vectors(*w.box)
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method("PME")
    nb.set_cutoff_distance(0.9)
    for q, sg, e in zip(w.charges(), w.sigmas(), w.epsilons()):
        nb.add_particle(float(q), float(sg), float(e))
    for ex in w.exceptions():
        nb.add_exception(*ex)
    nb.set_reciprocal_space_force_group(1)
    s.add_force(nb)
    ctx = ommb200.Context(s, systems.langevin(), precision="double")
    ctx.set_positions(w.positions)
    a = ctx.get_state(forces=True, energy=True)
    d = ctx.get_state(forces=True, energy=True, groups=1 << 0)
    r = ctx.get_state(forces=True, energy=True, groups=1 << 1)
    assert abs(d.potential_energy + r.potential_energy - a.potential_energy) < 1e-8 * abs(a.potential_energy)
    assert np.abs(d.forces + r.forces - a.forces).max() < 1e-8
    f_rec, e_rec = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                               method="PME", cutoff=0.9, box=w.box, include_direct=False)
    assert abs(r.potential_energy - e_rec) < 1e-8 * abs(e_rec)
    assert rms_rel(r.forces, f_rec) < 1e-9


# Grid shapes of the reciprocal part: odd and even axes, radices 2 to 8 in the engine's own
# transform, and prime factors 11, 13, 17 that take the cuFFT path.
@pytest.mark.parametrize("precision,bound", [("mixed", MIXED_FORCE_RMS), ("double", DOUBLE_FORCE_RMS)])
@pytest.mark.parametrize("grid", [(25, 27, 30), (32, 21, 28), (45, 35, 49), (16, 24, 20),
                                  (22, 26, 34), (5, 6, 7)])
def test_pme_grid_shapes_match_oracle(grid, precision, bound):
    w = synth.water_box(100, 2.0, (5, 5, 4), seed=4)
    s = ommb200.System()
    for m in w.masses():
        s.add_particle(float(m))
    s.set_default_periodic_box_vectors(*w.box)
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method("PME")
    nb.set_cutoff_distance(0.9)
    nb.set_pme_parameters(3.2, *grid)
    for q, sg, e in zip(w.charges(), w.sigmas(), w.epsilons()):
        nb.add_particle(float(q), float(sg), float(e))
    for ex in w.exceptions():
        nb.add_exception(*ex)
    nb.set_reciprocal_space_force_group(1)
    s.add_force(nb)
    ctx = ommb200.Context(s, systems.langevin(), precision=precision)
    ctx.set_positions(w.positions)
    r = ctx.get_state(forces=True, energy=True, groups=1 << 1)
    f_rec, e_rec = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                               method="PME", cutoff=0.9, box=w.box, include_direct=False,
                               pme=(3.2, grid))
    e_tol = 2e-6 if precision == "mixed" else 1e-9
    assert abs(r.potential_energy - e_rec) < e_tol * abs(e_rec)
    assert rms_rel(r.forces, f_rec) < bound


def test_nve_energy_is_conserved():
    """friction 0, temperature 0: LangevinMiddle reduces to velocity Verlet with SETTLE.  At the
    production 2 fs step over 40 ps (after 10 ps without the thermostat): the total energy
    fluctuates by well under 1 % of the kinetic energy, and its drift is below 0.1 kJ/mol/ns
    per degree of freedom (6 per rigid
    water; a thermostat-free run that heats or cools at that rate changes its temperature by
    about 12 K per ns; the 100 ps drift of the 23,958-atom box measured by bench.py is
    0.0002 +- 0.002)."""
    w, x, v = equilibrated_water()
    integ = ommb200.LangevinMiddleIntegrator(0.0, 0.0, 0.002)
    ctx = ommb200.Context(systems.water_system(w), integ, precision="mixed")
    ctx.set_positions(x)
    ctx.set_velocities(v)
    ctx.step(5000)  # let the thermostat-free state settle
    t, e = [], []
    for k in range(201):
        st = ctx.get_state(energy=True)
        t.append(0.2 * k)  # ps
        e.append(st.potential_energy + st.kinetic_energy)
        ctx.step(100)
    t, e = np.array(t), np.array(e)
    ke = ctx.get_state(energy=True).kinetic_energy
    assert np.abs(e - e.mean()).max() < 0.01 * ke, (e.max() - e.min(), ke)
    dof = 6 * w.n_waters
    slope = np.polyfit(t, e, 1)[0] * 1000.0 / dof  # kJ/mol/ns per degree of freedom
    assert abs(slope) < 0.1, slope
