"""The culling pair kernel (ommb200_options.pair_cull) against the f64 oracle and against the
kernel that evaluates every listed entry.

The culling kernel drops, at every force evaluation, the neighbour entries that lie beyond the
cutoff (plus the f64 decision band) of the current bounding box of their half block, and packs
the rest into full rounds.  The pair set must stay the reference's exactly (forces/neighbors.rs
cell pairs with r^2 < rc^2, nonbonded.rs:862); forces within the mixed-precision target of
5e-6 RMS relative error; runs bit-identical for the same inputs, whichever warps take which
runs of tiles.  Cases: the 1,944-atom box (small: neighbour tiles that take the minimum image
per pair), the 23,958-atom box, and a box with a third of its water sites empty (blocks with an
empty half, padding entries, uneven tile counts).
"""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import synth, systems

pytestmark = pytest.mark.gpu

MIXED_FORCE_RMS = 5e-6
CULL_RUNS = [1, 3, 8, 64]


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


_BOXES = {}


def box(name):
    if name not in _BOXES:
        if name == "sparse":
            w = synth.water_box(1150, 3.6, (12, 12, 12), seed=11)
        else:
            w = synth.water_preset(name)
        f, e, v = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(),
                              w.exceptions(), method="PME", cutoff=0.9, ewald_tolerance=5e-4,
                              box=w.box, threads=8, virial=True)
        _BOXES[name] = (w, f, e, v)
    return _BOXES[name]


def context(w, pair_cull, precision="mixed", **kw):
    ctx = ommb200.Context(systems.water_system(w), systems.langevin(seed=7), precision=precision,
                          pair_cull=pair_cull, **kw)
    ctx.set_positions(w.positions)
    return ctx


def pair_keys(pairs):
    return np.sort(pairs[:, 0].astype(np.int64) * 10_000_000 + pairs[:, 1])


@pytest.mark.parametrize("name", ["water-1944", "water-23958", "sparse"])
def test_culled_forces_energy_virial_match_oracle(name):
    w, f_ref, e_ref, vir_ref = box(name)
    plain = context(w, 0)
    assert plain.tuning()["cull_tiles"] == 0
    st0 = plain.get_state(forces=True, energy=True, virial=True)
    for k in CULL_RUNS:
        ctx = context(w, k)
        assert ctx.tuning()["cull_tiles"] == k
        st = ctx.get_state(forces=True, energy=True, virial=True)
        err = rms_rel(st.forces, f_ref)
        print(f"{name} cull {k}: force rms rel {err:.3e} (plain {rms_rel(st0.forces, f_ref):.3e})")
        assert err < MIXED_FORCE_RMS
        # the same pairs in other float groupings: the two kernels agree to rounding
        assert rms_rel(st.forces, st0.forces) < 1e-6
        assert abs(st.potential_energy - e_ref) < 2e-6 * abs(e_ref) + 1e-6 * w.n_atoms
        assert np.abs(st.virial - vir_ref).max() < 1e-4 * np.abs(vir_ref).max()


@pytest.mark.parametrize("name", ["water-1944", "water-23958", "sparse"])
def test_culled_pair_set_is_the_reference_pair_set(name):
    w = box(name)[0]
    ref = O.pair_set(w.positions, 0.9, box=w.box, exclusions=[e[:2] for e in w.exceptions()])
    for k in (1, 8, 64):
        got = context(w, k).debug_pair_list()
        assert len(got) == len(ref), (k, len(got), len(ref))
        assert np.array_equal(pair_keys(got), pair_keys(ref)), k


def test_culled_pair_set_after_dynamics_and_rebuilds():
    """Between rebuilds the particles move through the skin; the culling boxes follow the
    current positions, so every pair that comes within the cutoff is still met."""
    w = box("water-1944")[0]
    ctx = context(w, 8)
    ctx.set_velocities_to_temperature(300.0, seed=5)
    ctx.step(75)
    pos = ctx.get_state(positions=True).positions
    ref = O.pair_set(pos, 0.9, box=w.box, exclusions=[e[:2] for e in w.exceptions()])
    got = ctx.debug_pair_list()
    assert np.array_equal(pair_keys(got), pair_keys(ref))


@pytest.mark.parametrize("use_graph", [True, False])
def test_culled_dynamics_are_bit_identical_run_to_run(use_graph):
    """Runs of tiles are fetched by whichever warp is free; the forces of a run do not depend
    on which warp takes it, so two runs from the same state agree bit for bit."""
    w = box("sparse")[0]
    out = []
    for _ in range(2):
        ctx = context(w, 4, use_cuda_graph=use_graph)
        ctx.set_velocities_to_temperature(300.0, seed=3)
        ctx.step(60)
        st = ctx.get_state(positions=True, velocities=True, forces=True)
        out.append((st.positions.copy(), st.velocities.copy(), st.forces.copy()))
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)


def test_culling_applies_to_the_mixed_form_without_a_pruned_list_only():
    w = box("water-1944")[0]
    assert context(w, 8, precision="double").tuning()["cull_tiles"] == 0
    assert context(w, 8, prune_margin=0.05).tuning()["cull_tiles"] == 0
    # by size: a 1,944-atom list gives each warp a fraction of a tile, so it stays off
    assert context(w, -1).tuning()["cull_tiles"] == 0


@pytest.mark.parametrize("name", ["water-1944", "sparse"])
def test_culled_reaction_field_with_switching_matches_oracle(name):
    """The reaction-field form with an LJ switching function (nonbonded.rs:888-900,
    1222-1243) through the culling kernel: the same pairs, the same forces as the oracle."""
    w = box(name)[0]
    f_ref, e_ref = O.nonbonded(w.positions, w.charges(), w.sigmas(), w.epsilons(),
                               w.exceptions(), method="CutoffPeriodic", cutoff=0.9, box=w.box,
                               use_switching=True, switching_distance=0.8, threads=8)
    ref_pairs = O.pair_set(w.positions, 0.9, box=w.box,
                           exclusions=[e[:2] for e in w.exceptions()])
    for k in (0, 1, 8):
        ctx = ommb200.Context(systems.water_system(w, method="CutoffPeriodic",
                                                   switching_distance=0.8),
                              systems.langevin(seed=7), pair_cull=k)
        ctx.set_positions(w.positions)
        assert ctx.tuning()["cull_tiles"] == k
        st = ctx.get_state(forces=True, energy=True)
        assert rms_rel(st.forces, f_ref) < MIXED_FORCE_RMS, k
        # the reaction-field total is small (~1 kJ/mol per atom) beside the pair energies
        # it sums, so its FP32 error is bounded per atom rather than relative to the total
        assert abs(st.potential_energy - e_ref) < 2e-5 * w.n_atoms, k
        got = ctx.debug_pair_list()
        assert np.array_equal(pair_keys(got), pair_keys(ref_pairs)), k


def test_culled_checkpoint_continues_bit_for_bit():
    """The checkpoint carries the run length, so a Context created without culling continues a
    culled trajectory bit for bit."""
    w = box("sparse")[0]
    a = context(w, 8)
    a.set_velocities_to_temperature(300.0, seed=5)
    a.step(80)
    ck = a.create_checkpoint()
    a.step(60)
    sa = a.get_state(positions=True, velocities=True, forces=True, energy=True)
    b = context(w, 0)
    b.load_checkpoint(ck)
    assert b.tuning()["cull_tiles"] == 8
    b.step(60)
    sb = b.get_state(positions=True, velocities=True, forces=True, energy=True)
    assert np.array_equal(sa.positions, sb.positions)
    assert np.array_equal(sa.velocities, sb.velocities)
    assert np.array_equal(sa.forces, sb.forces)
    assert sa.potential_energy == sb.potential_energy
