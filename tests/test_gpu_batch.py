"""Batches of independent implicit-solvent chains in one Context: every System of the batch
gives the same forces, energies and (without noise) trajectory as its own Context, and the
forces match the f64 oracle.  A batch has no reference counterpart; the per-System terms it
evaluates are NonbondedForce (nonbonded.rs), GBSAOBCForce (gbsa_obc.rs), HarmonicBondForce
and HarmonicAngleForce, integrated by LangevinMiddleIntegrator (langevin.rs)."""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu

SIZES = [37, 200, 64, 513, 9]  # ragged: partial blocks, one exact block, one tiny system


def chains(sizes=SIZES, seed=3):
    return [synth.chain(n, seed=seed + k) for k, n in enumerate(sizes)]


def batch_context(chs, precision="mixed", cutoff=None, friction=1.0, **kw):
    sysms = [systems.chain_system(c, cutoff=cutoff, **kw) for c in chs]
    ctx = ommb200.BatchContext(sysms, systems.langevin(friction=friction, step_size=0.001, seed=5),
                               precision=precision)
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    return ctx


def single_context(ch, precision="mixed", cutoff=None, friction=1.0, **kw):
    ctx = ommb200.Context(systems.chain_system(ch, cutoff=cutoff, **kw),
                          systems.langevin(friction=friction, step_size=0.001, seed=5),
                          precision=precision)
    ctx.set_positions(ch.positions)
    return ctx


def oracle_forces(ch, cutoff=None):
    n = ch.n_atoms
    excl = sorted({(i, i + 1) for i in range(n - 1)} | {(i, i + 2) for i in range(n - 2)})
    exc = [(i, j, 0.0, ch.sigma, 0.0) for i, j in excl]
    exc += [(i, i + 3, ch.charges[i] * ch.charges[i + 3], ch.sigma, ch.epsilon)
            for i in range(n - 3)]
    if cutoff is None:
        f1, e1 = O.nonbonded(ch.positions, ch.charges, [ch.sigma] * n, [ch.epsilon] * n, exc,
                             method="NoCutoff")
        f4, e4, _ = O.gbsa_obc(ch.positions, ch.charges, ch.radii, [ch.gb_scale] * n,
                               solvent_dielectric=78.5, solute_dielectric=1.0)
    else:
        f1, e1 = O.nonbonded(ch.positions, ch.charges, [ch.sigma] * n, [ch.epsilon] * n, exc,
                             method="CutoffNonPeriodic", cutoff=cutoff)
        f4, e4, _ = O.gbsa_obc(ch.positions, ch.charges, ch.radii, [ch.gb_scale] * n, method=1,
                               cutoff=cutoff, solvent_dielectric=78.5, solute_dielectric=1.0)
    f2, e2 = O.harmonic_bonds(ch.positions, ch.bonds())
    f3, e3 = O.harmonic_angles(ch.positions, ch.angles())
    return f1 + f2 + f3 + f4, e1 + e2 + e3 + e4


def test_layout_and_ranges():
    chs = chains()
    ctx = batch_context(chs)
    assert ctx.num_systems() == len(SIZES)
    assert ctx.num_particles() == sum(SIZES)
    first = np.concatenate([[0], np.cumsum(SIZES)[:-1]])
    assert [ctx.system_range(k) for k in range(len(SIZES))] == list(zip(first, SIZES))
    with pytest.raises(ommb200.InvalidArgument):
        ctx.system_range(len(SIZES))


@pytest.mark.parametrize("cutoff", [None, 1.2])
@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_batch_equals_separate_contexts(precision, cutoff):
    """Forces and per-System energies are bit-identical to one Context per System: the batch
    pads each System to whole 32-slot blocks and sums the same fixed-point terms."""
    chs = chains()
    ctx = batch_context(chs, precision, cutoff)
    st = ctx.get_state(forces=True, energy=True)
    pot, _ = ctx.system_energies()
    for k, (ch, f) in enumerate(zip(chs, ctx.split(st.forces))):
        one = single_context(ch, precision, cutoff).get_state(forces=True, energy=True)
        assert np.array_equal(f, one.forces), k
        assert pot[k] == one.potential_energy, k
    assert abs(pot.sum() - st.potential_energy) <= 1e-9 * abs(st.potential_energy)


@pytest.mark.parametrize("cutoff", [None, 1.2])
@pytest.mark.parametrize("precision,bound", [("double", 1e-9), ("mixed", 5e-6)])
def test_batch_matches_oracle(precision, bound, cutoff):
    chs = chains()
    ctx = batch_context(chs, precision, cutoff)
    st = ctx.get_state(forces=True, energy=True)
    pot, _ = ctx.system_energies()
    for k, (ch, f) in enumerate(zip(chs, ctx.split(st.forces))):
        f_ref, e_ref = oracle_forces(ch, cutoff)
        err = float(np.sqrt(((f - f_ref) ** 2).sum() / (f_ref ** 2).sum()))
        assert err < bound, (k, err)
        etol = 1e-9 if precision == "double" else 2e-6
        assert abs(pot[k] - e_ref) < etol * abs(e_ref) + 1e-6, (k, pot[k], e_ref)


def test_group_selection_per_system():
    chs = chains()
    sysms = []
    for c in chs:
        s = systems.chain_system(c)
        sysms.append(s)
    ctx = ommb200.BatchContext(sysms, systems.langevin(step_size=0.001), precision="double")
    ctx.set_positions(np.concatenate([c.positions for c in chs]))
    pot_all, _ = ctx.system_energies()
    pot_none, _ = ctx.system_energies(groups=0)
    assert np.all(pot_none == 0.0)
    assert np.all(pot_all != 0.0)


def test_frictionless_trajectories_match_separate_contexts():
    """With friction 0 the Langevin noise term vanishes, so each System of the batch follows
    exactly the trajectory of its own Context (the random stream depends on the particle's
    index in the batch, which only matters with friction)."""
    chs = chains()
    rng = np.random.default_rng(11)
    vels = [rng.normal(0.0, 0.5, (c.n_atoms, 3)) for c in chs]
    ctx = batch_context(chs, friction=0.0)
    ctx.set_velocities(np.concatenate(vels))
    ctx.step(150)
    st = ctx.get_state(positions=True, velocities=True, energy=True)
    pot, kin = ctx.system_energies()
    for k, ch in enumerate(chs):
        one = single_context(ch, friction=0.0)
        one.set_velocities(vels[k])
        one.step(150)
        ref = one.get_state(positions=True, velocities=True, energy=True)
        assert np.array_equal(ctx.split(st.positions)[k], ref.positions), k
        assert np.array_equal(ctx.split(st.velocities)[k], ref.velocities), k
        assert pot[k] == ref.potential_energy, k
        assert abs(kin[k] - ref.kinetic_energy) <= 1e-12 * ref.kinetic_energy, k


def test_many_uneven_systems_thermostat():
    """A larger ragged batch stays finite and every System thermalises near 300 K."""
    chs = synth.chain_batch(24, lo=40, hi=300, seed=2)
    ctx = batch_context(chs, friction=10.0)
    ctx.set_velocities_to_temperature(300.0, seed=4)
    ctx.step(3000)
    st = ctx.get_state(positions=True, energy=True)
    assert np.isfinite(st.positions).all()
    _, kin = ctx.system_energies()
    dof = np.array([3 * c.n_atoms for c in chs])
    temps = 2.0 * kin / (dof * 0.008314462618)
    assert np.isfinite(temps).all()
    assert 250.0 < temps.mean() < 350.0, temps
