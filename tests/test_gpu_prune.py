"""The pruned pair list between rebuilds (periodic rectangular boxes).

After a rebuild, and again once a particle has moved half the prune margin, the engine cuts the
rebuild's tiles down to the entries within cutoff + margin of their half block; the pair kernel
reads that list until the next prune.  The interacting pair set must stay the reference's exact
set (nonbonded.rs: every pair within the cutoff, exclusions left out) at every step, including
steps where the last prune is several steps old, and the forces must stay the oracle's.
"""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu


def pair_keys(p):
    return np.sort(p[:, 0].astype(np.int64) * 10_000_000 + p[:, 1])


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_pair_set_between_prunes_is_the_reference_pair_set(precision):
    w = synth.water_preset("water-1944")
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(temperature=400.0, seed=13),
                          precision=precision, prune_margin=0.05)
    ctx.set_positions(w.positions)
    ctx.set_velocities_to_temperature(400.0, seed=6)
    excl = [e[:2] for e in w.exceptions()]
    seen_old_prune = 0
    for chunk in range(12):
        before = ctx.nlist_prune_stats()["prunes"]
        ctx.step(1 + chunk % 4)
        stats = ctx.nlist_prune_stats()
        assert stats["margin_nm"] > 0.0
        seen_old_prune += stats["prunes"] == before  # the list in use was pruned steps ago
        pos = ctx.get_state(positions=True).positions
        ref = O.pair_set(pos, 0.9, box=w.box, exclusions=excl)
        got = ctx.debug_pair_list()
        assert len(got) == len(ref), (chunk, len(got), len(ref))
        assert np.array_equal(pair_keys(got), pair_keys(ref)), chunk
    assert ctx.nlist_prune_stats()["prunes"] >= 3
    assert seen_old_prune >= 1
    ctx.close()


def test_pruned_list_is_smaller_and_forces_match_oracle():
    w = synth.water_preset("water-1944")
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(seed=17), precision="mixed",
                          prune_margin=0.08)
    ctx.set_positions(w.positions)
    ctx.set_velocities_to_temperature(300.0, seed=8)
    ctx.step(45)
    stats = ctx.nlist_prune_stats()
    tiles_in_use = ctx.nlist_stats()["tiles"]
    assert 0 < tiles_in_use < stats["rebuild_tiles"]
    st = ctx.get_state(positions=True, forces=True, energy=True)
    f_ref, e_ref = O.nonbonded(st.positions, w.charges(), w.sigmas(), w.epsilons(), w.exceptions(),
                               method="PME", cutoff=0.9, ewald_tolerance=5e-4, box=w.box,
                               threads=8)
    err = float(np.sqrt(((st.forces - f_ref) ** 2).sum() / (f_ref ** 2).sum()))
    assert err < 5e-6
    assert abs(st.potential_energy - e_ref) < 2e-6 * abs(e_ref) + 1e-6 * w.n_atoms
    ctx.close()


def test_pruning_is_off_by_default_and_margin_zero():
    w = synth.water_preset("water-1944")
    for kw in ({}, {"prune_margin": 0.0}):
        ctx = ommb200.Context(systems.water_system(w), systems.langevin(), **kw)
        ctx.set_positions(w.positions)
        ctx.step(5)
        assert ctx.nlist_prune_stats()["margin_nm"] == 0.0
        assert ctx.nlist_prune_stats()["prunes"] == 0
        ctx.close()
