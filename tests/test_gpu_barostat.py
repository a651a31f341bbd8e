"""MonteCarloBarostat through the C ABI (forces/barostat.rs, context/program.rs:5-47), checked
against the oracle's restatement of the move: scaled positions, the Metropolis work and test,
the volume-step adaptation, the energy change, and the reference's own barostat tests
(tests/barostat.rs) restated for this engine."""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu

TRICLINIC = [[3.0, 0.0, 0.0], [0.4, 4.0, 0.0], [-0.2, 0.3, 5.0]]
POS3 = np.array([[0.2, 0.3, 0.4], [0.9, 0.3, 0.4], [1.4, 1.1, 0.8]])


def bond_context(rigid=True, frequency=1, pressure=0.0, temperature=0.0, seed=47):
    # tests/barostat.rs:18-43: masses 1, 3, 0; a zero-stiffness periodic bond between 0 and 1
    s = ommb200.System()
    for m in (1.0, 3.0, 0.0):
        s.add_particle(m)
    s.set_default_periodic_box_vectors(*TRICLINIC)
    hb = ommb200.HarmonicBondForce()
    hb.add_bond(0, 1, 0.7, 0.0)
    hb.set_uses_periodic_boundary_conditions(True)
    s.add_force(hb)
    bar = ommb200.MonteCarloBarostat(pressure, temperature, frequency)
    bar.set_scale_molecules_as_rigid(rigid)
    bar.set_random_number_seed(seed)
    s.add_force(bar)
    ctx = ommb200.Context(s, ommb200.LangevinMiddleIntegrator(0.0, 0.0, 0.001), precision="double")
    ctx.set_positions(POS3)
    return ctx, bar


def box_and_positions(ctx):
    st = ctx.get_state(positions=True)
    return np.array(st.periodic_box_vectors), st.positions


@pytest.mark.parametrize("rigid", [True, False])
def test_scaling_matches_the_oracle_and_keeps_the_captured_mode(rigid):
    # tests/barostat.rs:58-84: zero energy change at zero pressure and temperature: accepted
    ctx, bar = bond_context(rigid=rigid)
    bar.set_scale_molecules_as_rigid(not rigid)  # taken at Context creation: no effect now
    ctx.step(1)
    box, after = box_and_positions(ctx)
    scale = box[0][0] / 3.0
    assert scale != 1.0
    st = ctx.barostat_stats()
    mols = O.molecules(3, bonds=[(0, 1)])
    move = np.cbrt(st["last_new_volume"] / st["last_old_volume"])
    expect = O.scale_positions(POS3, mols, move, rigid)
    assert np.abs(after - expect).max() < 2e-15
    assert st["attempted"] == 1 and st["accepted"] == 1 and st["last_accepted"] == 1
    assert np.allclose(box, np.array(TRICLINIC) * scale, rtol=0, atol=1e-15)


def test_rejection_preserves_coordinates_and_box():
    # tests/barostat.rs:149-167
    ctx, _ = bond_context()
    ctx.set_parameter(ommb200.MonteCarloBarostat.PRESSURE, 1e30)
    previous = 60.0
    for _ in range(50):
        ctx.step(1)
        box, pos = box_and_positions(ctx)
        volume = box[0][0] * box[1][1] * box[2][2]
        assert volume <= previous + 1e-12
        if volume == previous == 60.0:
            assert np.array_equal(pos, POS3)
        previous = volume
    assert previous < 60.0


def test_schedule_uses_its_own_counter_and_a_live_frequency():
    # tests/barostat.rs:86-107
    a, control = bond_context(frequency=0)
    b, _ = bond_context(frequency=1)
    box0, _ = box_and_positions(a)
    a.set_step_count(90)
    a.step(5)
    assert np.array_equal(box_and_positions(a)[0], box0)
    control.set_frequency(4)  # the Context holds this barostat: the change reaches it
    a.set_step_count(0)
    a.step(1)
    b.step(1)
    (ba, pa), (bb, pb) = box_and_positions(a), box_and_positions(b)
    assert not np.array_equal(ba, box0)
    assert np.array_equal(ba, bb) and np.array_equal(pa, pb)
    control.set_frequency(1)
    for _ in range(30):
        a.step(1)
        b.step(1)
        assert np.array_equal(box_and_positions(a)[0], box_and_positions(b)[0])


def test_invalid_volume_proposals_are_rejected_without_nonfinite_boxes():
    # barostat.rs:283-304: a 1 nm box gives a 0.01 nm^3 volume step; in a 0.01 nm box most
    # proposals have a negative volume
    s = ommb200.System()
    s.add_particle(1.0)
    s.set_default_periodic_box_vectors([1, 0, 0], [0, 1, 0], [0, 0, 1])
    hb = ommb200.HarmonicBondForce()
    hb.set_uses_periodic_boundary_conditions(True)
    s.add_force(hb)
    bar = ommb200.MonteCarloBarostat(1.0, 300.0, 1)
    bar.set_random_number_seed(13)
    s.add_force(bar)
    ctx = ommb200.Context(s, ommb200.LangevinMiddleIntegrator(0.0, 0.0, 0.001), precision="double")
    ctx.set_positions([[0.0, 0.0, 0.0]])
    ctx.set_periodic_box_vectors([0.01, 0, 0], [0, 0.01, 0], [0, 0, 0.01])
    ctx.step(100)
    st = ctx.barostat_stats()
    box, _ = box_and_positions(ctx)
    assert st["attempted"] == 100 and st["attempted"] - st["accepted"] > 10
    assert np.isfinite(box).all() and box[0][0] > 0.0


def test_water_moves_follow_the_metropolis_rule_and_the_energy_change():
    w = synth.water_preset("water-1944")
    s = systems.water_system(w)
    bar = ommb200.MonteCarloBarostat(1.0, 300.0, 1)
    bar.set_random_number_seed(5)
    s.add_force(bar)
    ctx = ommb200.Context(s, systems.langevin(seed=3), precision="double")
    ctx.set_positions(w.positions)
    ctx.set_velocities_to_temperature(300.0, seed=4)
    n_mol = len(O.molecules(w.n_atoms, constraints=[(i, j) for i, j, _ in w.constraints()]))
    assert n_mol == w.n_waters
    box0, _ = box_and_positions(ctx)
    step = O.VolumeStep(np.prod(np.diag(box0)))
    checked_energy = False
    for k in range(30):
        box_b, pos_b = box_and_positions(ctx)
        ctx.step(1)
        st = ctx.barostat_stats()
        v_old, v_new = st["last_old_volume"], st["last_new_volume"]
        assert abs(v_old - np.prod(np.diag(box_b))) < 1e-12 * v_old
        work = O.barostat_work(st["last_energy_change"], 1.0, v_old, v_new, n_mol, 300.0)
        assert abs(work - st["last_work"]) < 1e-9 * max(1.0, abs(work))
        acc = O.barostat_accepts(st["last_work"], 300.0, st["last_uniform"])
        assert acc == bool(st["last_accepted"])
        step.record(acc, v_old)
        assert abs(step.scale - st["volume_scale"]) < 1e-12 * step.scale
        box_a, _ = box_and_positions(ctx)
        assert abs(np.prod(np.diag(box_a)) - (v_new if acc else v_old)) < 1e-9 * v_old
        if not checked_energy:  # the energy change of this move from the oracle
            scale = np.cbrt(v_new / v_old)
            mols = O.molecules(w.n_atoms, constraints=[(i, j) for i, j, _ in w.constraints()])
            pos_s = O.scale_positions(pos_b, mols, scale, True)

            def energy(p, b):
                return O.nonbonded(p, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                                   method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=b,
                                   threads=8)[1]

            d_ref = energy(pos_s, box_b * scale) - energy(pos_b, box_b)
            assert abs(st["last_energy_change"] - d_ref) < 1e-8 * 3e4
            checked_energy = True
    assert st["attempted"] == 30


def test_npt_checkpoint_continues_bit_for_bit():
    w = synth.water_preset("water-1944")

    def make():
        s = systems.water_system(w)
        bar = ommb200.MonteCarloBarostat(1.0, 300.0, 5)
        bar.set_random_number_seed(11)
        s.add_force(bar)
        ctx = ommb200.Context(s, systems.langevin(seed=3))
        ctx.set_positions(w.positions)
        return ctx

    a = make()
    a.set_velocities_to_temperature(300.0, seed=2)
    a.step(23)
    ck = a.create_checkpoint()
    a.step(31)
    b = make()
    b.load_checkpoint(ck)
    b.step(31)
    (ba, pa), (bb, pb) = box_and_positions(a), box_and_positions(b)
    assert np.array_equal(ba, bb) and np.array_equal(pa, pb)
    assert a.barostat_stats() == b.barostat_stats()


def test_parameters_and_periodicity_are_validated():
    ctx, _ = bond_context(pressure=2.5, temperature=310.0)
    assert ctx.get_parameter(ommb200.MonteCarloBarostat.PRESSURE) == 2.5
    assert ctx.get_parameter(ommb200.MonteCarloBarostat.TEMPERATURE) == 310.0
    ctx.set_parameter(ommb200.MonteCarloBarostat.TEMPERATURE, 280.0)
    assert ctx.get_parameter(ommb200.MonteCarloBarostat.TEMPERATURE) == 280.0
    with pytest.raises(ommb200.InvalidArgument):
        ctx.set_parameter(ommb200.MonteCarloBarostat.TEMPERATURE, -1.0)
    with pytest.raises(ommb200.InvalidArgument):
        ctx.get_parameter("NoSuchParameter")
    # context.rs:95-101: a barostat needs a periodic System
    s = ommb200.System()
    s.add_particle(1.0)
    s.add_force(ommb200.MonteCarloBarostat(1.0, 300.0, 25))
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.Context(s, ommb200.LangevinMiddleIntegrator(300.0, 1.0, 0.001))


def test_graph_and_stream_paths_agree_with_volume_moves():
    # moves every 30 steps: the graph path runs 20-step graphs between moves and drops the
    # captured graph after every accepted move; it must follow the stream path bit for bit
    w = synth.water_preset("water-1944")
    out = []
    for graph in (True, False):
        s = systems.water_system(w)
        bar = ommb200.MonteCarloBarostat(1.0, 300.0, 30)
        bar.set_random_number_seed(21)
        s.add_force(bar)
        ctx = ommb200.Context(s, systems.langevin(seed=9), use_cuda_graph=graph)
        ctx.set_positions(w.positions)
        ctx.set_velocities_to_temperature(300.0, seed=6)
        ctx.step(200)
        out.append((box_and_positions(ctx), ctx.barostat_stats()))
    (ba, pa), sa = out[0]
    (bb, pb), sb = out[1]
    assert sa["attempted"] == sb["attempted"] == 6
    assert np.array_equal(ba, bb) and np.array_equal(pa, pb) and sa == sb
