"""C-ABI contract tests that need no GPU: the library loads, exports every entry point that
include/ommb200.h declares, validates arguments like the reference's asserts, and fails loudly
(no CPU fallback) when no CUDA device is present."""
import ctypes as C
import re
from pathlib import Path

import pytest

import ommb200
from ommb200 import synth, systems

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "ommb200.h").read_text()
    return sorted(set(re.findall(r"\b(ommb200_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ommb200.library()
    names = declared_symbols()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert "sm_100a" in ommb200.version()


@pytest.mark.parametrize("call", [
    lambda f: f.set_cutoff_distance(-1.0),
    lambda f: f.set_cutoff_distance(float("inf")),
    lambda f: f.set_ewald_error_tolerance(0.6),
    lambda f: f.set_reaction_field_dielectric(0.5),
    lambda f: f.set_switching_distance(-0.1),
    lambda f: f.set_pme_parameters(2.0, 4, 10, 10),
    lambda f: f.set_reciprocal_space_force_group(32),
    lambda f: f.add_particle(0.0, -1.0, 0.0),
    lambda f: f.add_particle(float("nan"), 0.3, 0.1),
    lambda f: f.set_nonbonded_method("Bogus"),
    lambda f: f.set_force_group(40),
])
def test_nonbonded_setters_validate_like_the_reference(call):
    # nonbonded.rs:111-611 asserts become InvalidArgument (or KeyError for unknown names)
    f = ommb200.NonbondedForce()
    with pytest.raises((ommb200.InvalidArgument, KeyError)):
        call(f)


def test_nonbonded_parameter_roundtrip():
    f = ommb200.NonbondedForce()
    assert f.add_particle(0.5, 0.3, 0.2) == 0
    assert f.add_particle(-0.5, 0.31, 0.21) == 1
    f.set_particle_parameters(1, -0.4, 0.32, 0.22)
    assert f.get_particle_parameters(1) == (-0.4, 0.32, 0.22)
    assert f.num_particles() == 2
    assert f.add_exception(0, 1, 0.0, 0.3, 0.0) == 0
    assert f.num_exceptions() == 1


def test_exceptions_from_bonds_matches_reference_rule():
    # nonbonded.rs:434-500 on a 6-atom chain: 1-2 and 1-3 excluded, 1-4 scaled
    f = ommb200.NonbondedForce()
    for q in [0.1, -0.2, 0.3, -0.1, 0.2, -0.3]:
        f.add_particle(q, 0.3, 0.4)
    f.create_exceptions_from_bonds([(i, i + 1) for i in range(5)], 0.5, 0.25)
    assert f.num_exceptions() == 5 + 4 + 3


def test_integrator_validation():
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.LangevinMiddleIntegrator(-1.0, 1.0, 0.002)
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.LangevinMiddleIntegrator(300.0, 1.0, 0.0)
    i = ommb200.LangevinMiddleIntegrator(300.0, 1.0, 0.002)
    with pytest.raises(ommb200.InvalidArgument):
        i.set_constraint_tolerance(1.5)


def test_box_must_be_reduced():
    s = ommb200.System()
    with pytest.raises(ommb200.InvalidArgument):
        s.set_default_periodic_box_vectors([2, 0.1, 0], [0, 2, 0], [0, 0, 2])
    with pytest.raises(ommb200.InvalidArgument):
        s.set_default_periodic_box_vectors([2, 0, 0], [1.5, 2, 0], [0, 0, 2])


def test_force_ownership_moves_into_system():
    s = ommb200.System()
    s.add_particle(1.0)
    f = ommb200.NonbondedForce()
    f.add_particle(0.0, 0.3, 0.1)
    assert s.add_force(f) == 0
    with pytest.raises(ommb200.InvalidArgument):
        s.add_force(f)


def test_context_creation_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    w = synth.water_box(8, 1.9, (2, 2, 2), seed=1)
    s = systems.water_system(w)
    with pytest.raises(ommb200.OmmB200Error) as e:
        ommb200.Context(s, systems.langevin())
    assert e.value.code == ommb200.ERR_CUDA


def test_header_status_codes_match_python():
    text = (ROOT / "include" / "ommb200.h").read_text()
    codes = dict(re.findall(r"#define OMMB200_(ERR_[A-Z_]+) \((-\d+)\)", text))
    for name, value in codes.items():
        assert getattr(ommb200, name) == int(value), name


def test_batch_validation_happens_before_the_device():
    """Batch creation checks its Systems on the host: mismatched force kinds or settings and
    periodic Systems are refused with their own codes (no GPU is touched)."""
    chs = [synth.chain(20, seed=1), synth.chain(30, seed=2)]
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.BatchContext([systems.chain_system(chs[0]),
                              systems.chain_system(chs[1], gbsa=False)], systems.langevin())
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.BatchContext([systems.chain_system(chs[0]),
                              systems.chain_system(chs[1], cutoff=1.0)], systems.langevin())
    w = synth.water_box(8, 1.9, (2, 2, 2), seed=1)
    with pytest.raises(ommb200.OmmB200Error) as e:
        ommb200.BatchContext([systems.water_system(w), systems.water_system(w)],
                             systems.langevin())
    assert e.value.code == ommb200.ERR_UNSUPPORTED
    s = systems.chain_system(chs[0])
    with pytest.raises(ommb200.InvalidArgument):
        ommb200.BatchContext([s, s], systems.langevin())  # the second take is refused
    lib = ommb200.library()
    h = C.c_void_p()
    integ = systems.langevin()
    assert lib.ommb200_context_create_batch(None, 0, integ._take(), None, C.byref(h)) == \
        ommb200.ERR_INVALID_ARG


def test_default_options_and_option_validation():
    """ommb200_default_options fills the layout options (pme_bricks -1: by grid size;
    prune_margin -1: the default, no pruned list; pair_cull -1: the default run length of the
    culling pair kernel), and out-of-range values are refused before any device work, with or
    without a GPU."""
    opt = ommb200.Options()
    ommb200.library().ommb200_default_options(C.byref(opt))
    assert opt.use_cuda_graph == 1 and opt.steps_per_graph == 0
    assert opt.pme_bricks == -1 and opt.prune_margin == -1.0 and opt.pair_cull == -1
    w = synth.water_box(8, 1.9, (2, 2, 2), seed=1)
    for kw in ({"pme_bricks": 2}, {"prune_margin": 0.8}, {"prune_margin": float("nan")},
               {"pair_cull": -2}, {"pair_cull": 65}):
        with pytest.raises(ommb200.InvalidArgument):
            ommb200.Context(systems.water_system(w), systems.langevin(), **kw)
