"""Error paths of the engine, each failure made on the host (no GPU fault, no endless wait).

The reference's contract for a failed step is an error returned without corrupting the state
(constraints.rs:88-155, tests/constraints.rs:77-97).  Here:
* a neighbour list that overflows (a periodic box with one column far denser than the mean)
  grows and recovers: the forces equal the oracle's, and a batch of steps that overflows is
  re-run from its start to the trajectory of a Context whose list had grown beforehand;
* an infinite host-set velocity makes the dynamics nonfinite: the step reports NonfiniteError
  and the Context steps normally once finite positions and velocities are set again;
* a tensor-core wait that runs out (its poll limit set to zero) reports OMMB200_ERR_TIMEOUT,
  its kernel returns with the tensor memory freed, and the next call gives the oracle's values.
"""
import numpy as np
import pytest

import oracle as O
import ommb200
from ommb200 import systems

pytestmark = pytest.mark.gpu

BOX = 3.0
CUTOFF = 0.9


def dense_column_system(seed=3):
    """A periodic 3 nm box: a jittered 0.3 nm lattice outside one x-y corner column and a
    jittered 0.1 nm lattice (about 1,000 particles) inside it, ten times denser than the rest.
    Charges +-0.2 e, no LJ (reaction-field cutoff 0.9 nm)."""
    rng = np.random.default_rng(seed)
    g = (np.arange(10) + 0.5) * 0.3
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    lat = lat[~((lat[:, 0] < 0.65) & (lat[:, 1] < 0.65))]
    c = (np.arange(6) + 0.5) * 0.1
    z = (np.arange(30) + 0.5) * 0.1
    col = np.stack(np.meshgrid(c, c, z, indexing="ij"), -1).reshape(-1, 3)
    pos = np.vstack([lat, col]) + rng.uniform(-0.015, 0.015, (len(lat) + len(col), 3))
    n = len(pos)
    q = np.where(np.arange(n) % 2 == 0, 0.2, -0.2)
    sysm = ommb200.System()
    sysm.set_default_periodic_box_vectors([BOX, 0, 0], [0, BOX, 0], [0, 0, BOX])
    nb = ommb200.NonbondedForce()
    nb.set_nonbonded_method("CutoffPeriodic")
    nb.set_cutoff_distance(CUTOFF)
    for qi in q:
        sysm.add_particle(16.0)
        nb.add_particle(float(qi), 0.1, 0.0)
    sysm.add_force(nb)
    return sysm, pos, q


def oracle_forces(pos, q):
    f, e = O.nonbonded(pos, q, np.full(len(q), 0.1), np.zeros(len(q)), [],
                       method="CutoffPeriodic", cutoff=CUTOFF, box=np.eye(3) * BOX, threads=8)
    return f, e


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("pair_cull", [0, 8])
def test_overflowing_neighbor_list_grows_and_matches_the_oracle(pair_cull):
    sysm, pos, q = dense_column_system()
    ctx = ommb200.Context(sysm, systems.langevin(), precision="mixed", pair_cull=pair_cull)
    before = ctx.nlist_capacity()
    ctx.set_positions(pos)
    st = ctx.get_state(forces=True, energy=True)
    after = ctx.nlist_capacity()
    f_ref, e_ref = oracle_forces(pos, q)
    print(before, after, rms_rel(st.forces, f_ref))
    assert after["regrows"] >= 1
    assert after["column_capacity"] > before["column_capacity"]
    assert rms_rel(st.forces, f_ref) < 5e-6
    assert abs(st.potential_energy - e_ref) < 1e-5 * abs(e_ref) + 1e-3


@pytest.mark.parametrize("pair_cull", [0, 8])
def test_steps_that_overflow_rerun_to_the_grown_list_trajectory(pair_cull):
    """Also with the culling pair kernel: its runs are fixed slices of each block's own tiles,
    which do not depend on the list's capacity."""
    sysm, pos, q = dense_column_system()
    grown = ommb200.Context(sysm, systems.langevin(step_size=0.001, seed=9), precision="mixed",
                            pair_cull=pair_cull)
    grown.set_positions(pos)
    grown.set_velocities_to_temperature(300.0, seed=4)  # evaluates forces: the list grows here
    assert grown.nlist_capacity()["regrows"] >= 1
    v0 = grown.get_state(velocities=True).velocities
    sysm, _, _ = dense_column_system()  # a Context takes its System over
    fresh = ommb200.Context(sysm, systems.langevin(step_size=0.001, seed=9), precision="mixed",
                            pair_cull=pair_cull)
    fresh.set_positions(pos)
    fresh.set_velocities(v0)  # no force evaluation before the steps
    assert fresh.nlist_capacity()["regrows"] == 0
    grown.step(25)  # one captured group of 20 steps and 5 single steps
    fresh.step(25)  # overflows in its first batch, grows, restores and runs it again
    assert fresh.nlist_capacity()["regrows"] >= 1
    a = grown.get_state(positions=True, velocities=True, forces=True)
    b = fresh.get_state(positions=True, velocities=True, forces=True)
    assert np.array_equal(a.positions, b.positions)
    assert np.array_equal(a.velocities, b.velocities)
    assert a.step_count == b.step_count == 25
    f_ref, _ = oracle_forces(b.positions, q)
    assert rms_rel(b.forces, f_ref) < 5e-6


def test_nonfinite_dynamics_report_and_the_context_recovers():
    rng = np.random.default_rng(2)
    n = 64
    pos = rng.uniform(0.0, 2.0, (n, 3))
    sysm = ommb200.System()
    nb = ommb200.NonbondedForce()
    for i in range(n):
        sysm.add_particle(12.0)
        nb.add_particle(0.1 if i % 2 else -0.1, 0.3, 0.5)
    sysm.add_force(nb)
    ctx = ommb200.Context(sysm, systems.langevin(), precision="mixed")
    ctx.set_positions(pos)
    vel = np.zeros((n, 3))
    vel[5, 0] = np.inf
    ctx.set_velocities(vel)
    with pytest.raises(ommb200.NonfiniteError) as err:
        ctx.step(1)
    assert err.value.code == ommb200.ERR_NONFINITE
    ctx.set_positions(pos)
    ctx.set_velocities(np.zeros((n, 3)))
    ctx.step(5)
    st = ctx.get_state(positions=True, velocities=True, energy=True)
    assert np.isfinite(st.positions).all() and np.isfinite(st.velocities).all()
    assert np.isfinite(st.potential_energy)


def test_tensor_core_wait_timeout_reports_and_the_next_call_succeeds():
    torch = pytest.importorskip("torch")
    from test_gpu_radii_mlp import dev, random_params, synthetic_features

    rng = np.random.default_rng(21)
    g = synthetic_features(rng, 300)
    p = random_params(rng, g)
    ommb200.set_tensor_core_wait_limit(0)  # every MMA wait gives up at once
    try:
        with pytest.raises(ommb200.OmmB200Error) as err:
            ommb200.radii_mlp_forward(dev(g), dev(p))
        assert err.value.code == ommb200.ERR_TIMEOUT
    finally:
        ommb200.set_tensor_core_wait_limit(-1)
    tail, dt = ommb200.radii_mlp_forward(dev(g), dev(p))
    torch.cuda.synchronize()
    y, cache = O.mlp_forward(p, g)
    P = O.mlp_unpack(p)
    ref = y * float(P["t_scale"]) + float(P["t_mean"])
    err_y = np.abs(tail.cpu().numpy().astype(np.float64) - ref) / float(P["t_scale"])
    assert err_y.max() < 2e-2
