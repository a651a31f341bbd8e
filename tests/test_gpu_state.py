"""Checkpoints and live parameter updates (context.rs:274-293 set_state, context.rs:680-705
update_{gbsa_obc,nonbonded}_force_parameters): a checkpoint loaded into a fresh Context
continues the trajectory bit for bit, random stream and neighbour list included; updated
parameters give the forces of a Context built with them."""
import numpy as np
import pytest

import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu


def water_ctx(w, seed=3, prune_margin=-1.0, **kw):
    ctx = ommb200.Context(systems.water_system(w, **kw), systems.langevin(seed=seed),
                          prune_margin=prune_margin)
    ctx.set_positions(w.positions)
    return ctx


@pytest.mark.parametrize("margin", [0.0, 0.05])
def test_checkpoint_continues_water_bit_for_bit(margin):
    """With the pruned list (margin 0.05 nm) too: the loading Context starts without one and
    takes the margin, the prune positions and the pending-prune flag from the checkpoint."""
    w = synth.water_preset("water-1944")
    a = water_ctx(w, prune_margin=margin)
    a.set_velocities_to_temperature(300.0, seed=5)
    a.step(150)
    ck = a.create_checkpoint()
    a.step(170)
    sa = a.get_state(positions=True, velocities=True, forces=True, energy=True)
    stats_a = a.nlist_stats()
    b = water_ctx(w, seed=99)  # a different seed: the checkpoint carries the stream's
    b.load_checkpoint(ck)
    b.step(170)
    sb = b.get_state(positions=True, velocities=True, forces=True, energy=True)
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.velocities, sb.velocities)
    assert np.array_equal(sa.forces, sb.forces)
    assert sa.potential_energy == sb.potential_energy
    assert sa.step_count == sb.step_count == 320
    assert abs(sa.time - sb.time) < 1e-12
    assert stats_a["tiles"] == b.nlist_stats()["tiles"]
    assert a.nlist_prune_stats()["margin_nm"] == b.nlist_prune_stats()["margin_nm"] == margin


def test_checkpoint_continues_learned_radii_batch_bit_for_bit():
    chs = [synth.chain(400, seed=61), synth.chain(250, seed=62)]
    learned = {"judge_interval": 10, "train_steps": 4}

    def make():
        ctx = ommb200.BatchContext([systems.chain_system(c, learned_radii=learned) for c in chs],
                                   systems.langevin(step_size=0.001, seed=8))
        ctx.set_positions(np.concatenate([c.positions for c in chs]))
        return ctx

    a = make()
    a.set_velocities_to_temperature(300.0, seed=2)
    a.step(95)  # mid-interval: the next judge comes after the checkpoint
    ck = a.create_checkpoint()
    a.step(60)
    sa = a.get_state(positions=True, velocities=True)
    b = make()
    b.load_checkpoint(ck)
    b.step(60)
    sb = b.get_state(positions=True, velocities=True)
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.velocities, sb.velocities)
    assert np.array_equal(a.get_radii_mlp_params(), b.get_radii_mlp_params())
    assert a.learned_radii_stats() == b.learned_radii_stats()


def test_checkpoint_of_another_system_is_refused():
    w = synth.water_preset("water-1944")
    ck = water_ctx(w).create_checkpoint()
    ch = synth.chain(100, seed=1)
    other = ommb200.Context(systems.chain_system(ch), systems.langevin())
    other.set_positions(ch.positions)
    with pytest.raises(ommb200.InvalidArgument):
        other.load_checkpoint(ck)
    with pytest.raises(ommb200.InvalidArgument):
        water_ctx(w).load_checkpoint(ck[:100])


def _scaled_water_force(w, q_scale, eps_scale):
    nb = ommb200.NonbondedForce()
    for q, s, e in zip(w.charges(), w.sigmas(), w.epsilons()):
        nb.add_particle(float(q) * q_scale, float(s), float(e) * eps_scale)
    for i, j, qq, s, e in w.exceptions():
        nb.add_exception(i, j, qq, s, e)
    return nb


def test_nonbonded_update_matches_a_context_built_with_the_new_parameters():
    w = synth.water_preset("water-1944")
    ctx = water_ctx(w)
    ctx.update_nonbonded_parameters(_scaled_water_force(w, 0.9, 1.3))
    got = ctx.get_state(forces=True, energy=True)

    class Scaled:  # the same box with the parameters built in
        def __init__(self, w):
            self.w = w

        def __getattr__(self, k):
            return getattr(self.w, k)

        def charges(self):
            return self.w.charges() * 0.9

        def epsilons(self):
            return self.w.epsilons() * 1.3

    ref = water_ctx(Scaled(w)).get_state(forces=True, energy=True)
    assert np.array_equal(got.forces, ref.forces)
    assert got.potential_energy == ref.potential_energy


def test_nonbonded_update_keeps_exclusions():
    w = synth.water_preset("water-1944")
    ctx = water_ctx(w)
    nb = ommb200.NonbondedForce()
    for q, s, e in zip(w.charges(), w.sigmas(), w.epsilons()):
        nb.add_particle(float(q), float(s), float(e))
    exc = list(w.exceptions())
    for k, (i, j, qq, s, e) in enumerate(exc):
        nb.add_exception(i, j, 0.1 if k == 0 else qq, s, e)  # un-excluding the first pair
    with pytest.raises(ommb200.InvalidArgument):
        ctx.update_nonbonded_parameters(nb)
    short = ommb200.NonbondedForce()
    short.add_particle(0.0, 0.3, 0.1)
    with pytest.raises(ommb200.InvalidArgument):
        ctx.update_nonbonded_parameters(short)


def test_gbsa_update_matches_a_context_built_with_the_new_parameters():
    ch = synth.chain(300, seed=17)
    ctx = ommb200.Context(systems.chain_system(ch), systems.langevin(step_size=0.001))
    ctx.set_positions(ch.positions)
    new_r = ch.radii * 1.1
    gb = ommb200.GBSAOBCForce()
    for q, r in zip(ch.charges, new_r):
        gb.add_particle(float(q) * 0.8, float(r), ch.gb_scale)
    ctx.update_gbsa_obc_parameters(gb)
    got = ctx.get_state(forces=True, energy=True)
    ch2 = synth.Chain(positions=ch.positions, charges=ch.charges, radii=new_r)
    ref_sys = systems.chain_system(ch2)
    ref = ommb200.Context(ref_sys, systems.langevin(step_size=0.001))
    ref.set_positions(ch.positions)
    # only the GB charges were scaled: rebuild that part of the reference by hand
    ref_gb_only = ommb200.Context(_gb_system(ch, ch.charges * 0.8, new_r),
                                  systems.langevin(step_size=0.001))
    ref_gb_only.set_positions(ch.positions)
    base_gb_only = ommb200.Context(_gb_system(ch, ch.charges, new_r),
                                   systems.langevin(step_size=0.001))
    base_gb_only.set_positions(ch.positions)
    expect = (ref.get_state(forces=True).forces - base_gb_only.get_state(forces=True).forces +
              ref_gb_only.get_state(forces=True).forces)
    assert np.abs(got.forces - expect).max() < 1e-6 * np.abs(expect).max()


def _gb_system(ch, charges, radii):
    s = ommb200.System()
    gb = ommb200.GBSAOBCForce()
    gb.set_solvent_dielectric(78.5)
    gb.set_solute_dielectric(1.0)
    for q, r in zip(charges, radii):
        s.add_particle(ch.mass)
        gb.add_particle(float(q), float(r), ch.gb_scale)
    s.add_force(gb)
    return s
