"""The TOML reader follows the reference's input schema: includes, file_name
tables, env variables, offsets, defaults and its error cases; a system written
out and read back gives the oracle the same forces, energies and lists as the
golden fixtures made by the reference."""
import os
import textwrap

import numpy as np
import pytest

import oracle
from conftest import golden_cases
from mjolnir_b200 import input as I
from mjolnir_b200 import systems as S

CASES = golden_cases()


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(textwrap.dedent(text))
    return str(p)


@pytest.mark.parametrize("name", sorted(CASES))
def test_written_input_reproduces_golden(name, tmp_path):
    d, fx = CASES[name]
    path = str(tmp_path / "in.toml")
    I.dump(d, path)
    got = I.load(path).desc
    assert np.array_equal(got.pos, d.pos) and np.array_equal(got.vel, d.vel)
    o = oracle.Oracle(got)
    for t in ("bond", "angle", "dihedral", "exv", "dh", "lj"):
        if f"force_{t}" in fx:
            f, e = o.term_force(t, got.pos)
            ref = fx[f"force_{t}"]
            assert np.abs(f - ref).max() <= 1e-14 * max(np.abs(ref).max(), 1e-300), (name, t)
            assert e == pytest.approx(float(fx[f"energy_{t}"]), rel=1e-14, abs=1e-300)
        if f"pairs_{t}" in fx:
            assert np.array_equal(o.neighbors(t, got.pos), fx[f"pairs_{t}"].astype(np.int64)), (name, t)


def test_round_trip_keeps_every_field(tmp_path):
    d = S.polymer_melt(nchains=3, nbeads=12, radius=40.0, seed=5)
    path = str(tmp_path / "melt.toml")
    I.dump(d, path, total_step=500, save_step=50)
    inp = I.load(path)
    g = inp.desc
    assert (inp.total_step, inp.save_step, inp.precision) == (500, 50, "double")
    assert g.boundary == "Unlimited" and g.integrator == "BAOAB" and g.seed == d.seed
    assert g.dt == d.dt and g.temperature == d.temperature and g.ionic_strength == d.ionic_strength
    np.testing.assert_array_equal(g.mass, d.mass)
    np.testing.assert_array_equal(g.gamma, d.gamma)
    for a, b in ((g.bonds, d.bonds), (g.angles, d.angles), (g.dihedrals, d.dihedrals)):
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    for key in ("exv", "dh"):
        ta, tb = getattr(g, key), getattr(d, key)
        np.testing.assert_array_equal(ta.idx, tb.idx)
        np.testing.assert_array_equal(ta.param0, tb.param0)
        assert (ta.cutoff, ta.margin, ta.epsilon) == (tb.cutoff, tb.margin, tb.epsilon)
    assert g.ignore_molecule == "Nothing" and g.ignore_bond_within == 3


SIM = """
[simulator]
type          = "MolecularDynamics"
boundary_type = "PeriodicCuboid"
precision     = "double"
parallelism   = "OpenMP"
seed          = 2374
delta_t       = 0.005
total_step    = 100
save_step     = 10
integrator.type = "BAOABLangevin"
integrator.env.g = 1.0
integrator.gammas = [
{index = 0, gamma = "g"},
{index = 0, offset = 1, gamma = 0.5},
{index = 2, "γ" = 2.0},
{index = 3, gamma = 1.0},
]
"""

SYSTEM = """
[[systems]]
attributes.temperature = 300.0
boundary_shape.lower = [0.0, 0.0, 0.0]
boundary_shape.upper = [10.0, 10.0, 10.0]
particles = [
{mass = 1.0, position = [1.0, 1.0, 1.0]},
{m    = 2.0, pos      = [2.5, 1.0, 1.0]},
{mass = 1.0, position = [11.0, 1.0, -1.0]},
{mass = 1.0, position = [5.0, 5.0, 5.0], name = "C", group = "NONE"},
]
"""

FF = """
[[forcefields]]
[[forcefields.local]]
interaction = "BondLength"
potential   = "Harmonic"
topology    = "bond"
env.k = 10.0
parameters  = [
{indices = [0, 1], k = "k", v0 = 1.5},
{indices = [0, 1], offset = 1, k = 10.0, v0 = 1.5},
]
[[forcefields.global]]
interaction = "Pair"
potential   = "LennardJones"
ignore.molecule = "Nothing"
ignore.particles_within.bond = 1
spatial_partition = {type = "CellList", margin = 0.25}
env.s = 1.0
parameters = [
{index = 0, sigma = "s", epsilon = 1.0},
{index = 1, "σ" = 1.0, "ε" = 0.5},
{index = 1, offset = 1, sigma = 1.0, epsilon = 1.0},
{index = 3, sigma = 1.0, epsilon = 1.0},
]
"""

HEAD = """
[files]
output.prefix = "t"
output.path   = "./"
output.format = "xyz"
input.path    = "{path}"

[units]
length = "angstrom"
energy = "kcal/mol"
"""


def test_env_offsets_defaults_and_wrapping(tmp_path):
    path = _write(tmp_path, "in.toml", HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF)
    inp = I.load(path)
    d = inp.desc
    assert inp.parallelism == "OpenMP" and inp.seed == 2374 and d.seed == 2374
    np.testing.assert_array_equal(d.gamma, [1.0, 0.5, 2.0, 1.0])
    np.testing.assert_array_equal(d.mass, [1.0, 2.0, 1.0, 1.0])
    np.testing.assert_array_equal(d.pos[2], [1.0, 1.0, 9.0])       # wrapped into the box
    np.testing.assert_array_equal(d.bonds[0], [[0, 1], [1, 2]])
    np.testing.assert_array_equal(d.bonds[1], [10.0, 10.0])
    assert d.lj.cutoff == 2.5 and d.lj.margin == 0.25                # default LJ cutoff
    np.testing.assert_array_equal(d.lj.idx, [0, 1, 2, 3])
    np.testing.assert_array_equal(d.lj.param1, [1.0, 0.5, 1.0, 1.0])
    assert d.ignore_bond_within == 1
    # no velocities given: Maxwell-Boltzmann draws from the seed, reproducibly
    assert np.all(np.isfinite(d.vel)) and np.any(d.vel != 0)
    np.testing.assert_array_equal(I.load(path).desc.vel, d.vel)


def test_include_and_file_name(tmp_path):
    _write(tmp_path, "sim.toml", SIM.replace("[simulator]", ""))
    _write(tmp_path, "sys.toml", SYSTEM)
    _write(tmp_path, "ff.toml", FF.replace("[[forcefields]]", "").replace("[[forcefields.local]]", "[[local]]")
           .replace("[[forcefields.global]]", "[[global]]"))
    main = HEAD.format(path=str(tmp_path) + "/") + """
[simulator]
include = "sim.toml"
[[systems]]
file_name = "sys.toml"
[[forcefields]]
include = "ff.toml"
"""
    path = _write(tmp_path, "main.toml", main)
    d = I.load(path).desc
    flat = I.load(_write(tmp_path, "flat.toml", HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF)).desc
    np.testing.assert_array_equal(d.pos, flat.pos)
    np.testing.assert_array_equal(d.bonds[0], flat.bonds[0])
    np.testing.assert_array_equal(d.lj.param0, flat.lj.param0)


@pytest.mark.parametrize("edit, msg", [
    (lambda t: t.replace('potential   = "LennardJones"', 'potential   = "InversePower"'), "InversePower"),
    (lambda t: t.replace('ignore.molecule = "Nothing"', 'ignore.molecule = "Nothing"\nignore.group.intra = ["A"]'),
     "ignore.group"),
    (lambda t: t.replace('length = "angstrom"', 'length = "nm"'), "angstrom"),
    (lambda t: t.replace('{index = 3, sigma', '{index = 2, sigma'), "twice"),
    (lambda t: t.replace('{mass = 1.0, position = [1.0, 1.0, 1.0]}',
                         '{mass = 1.0, position = [1.0, 1.0, 1.0], velocity = [0.0, 0.0, 0.0]}'), "velocity"),
    (lambda t: t.replace('integrator.type = "BAOABLangevin"', 'integrator.type = "gBAOABLangevin"'),
     "BAOABLangevin"),
    (lambda t: t.replace('k = "k"', 'k = "kk"'), "kk"),
    (lambda t: t.replace('type = "CellList"', 'type = "Naive"'), "CellList"),
    (lambda t: t.replace('[0, 1], offset = 1', '[0, 7], offset = 1'), "out of range"),
])
def test_errors_name_the_problem(tmp_path, edit, msg):
    text = edit(HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF)
    path = _write(tmp_path, "bad.toml", text)
    with pytest.raises(I.InputError, match=msg):
        I.load(path)


def test_per_term_ignore_rules(tmp_path):
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF + """
[[forcefields.global]]
interaction = "Pair"
potential   = "DebyeHuckel"
ignore.molecule = "Self"
spatial_partition = {type = "VerletList", margin = 0.5}
parameters = [{index = 0, charge = 1.0}, {index = 3, charge = -1.0}]
"""
    text = text.replace("attributes.temperature = 300.0",
                        "attributes.temperature = 300.0\nattributes.ionic_strength = 0.1")
    d = I.load(_write(tmp_path, "in.toml", text)).desc
    assert d.dh.ignore_molecule == "Self" and d.dh.ignore_within == {}
    assert d.lj.ignore_molecule == "Nothing" and d.lj.ignore_within == {"bond": 1}
    assert d.dh.cutoff == 5.5
    with pytest.raises(NotImplementedError):
        oracle.make_spec(d)


def test_simulated_annealing_input(tmp_path):
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF
    text = text.replace('type          = "MolecularDynamics"', 'type          = "SimulatedAnnealing"')
    text = text.replace('save_step     = 10', 'save_step     = 10\neach_step     = 5\n'
                        'schedule = {type = "linear", begin = 350.0, end = 280.0}')
    inp = I.load(_write(tmp_path, "anneal.toml", text))
    assert inp.simulator == "SimulatedAnnealing" and inp.schedule == (350.0, 280.0, 5)
    assert inp.desc.temperature == 350.0            # current(0) before initialisation
    with pytest.raises(I.InputError, match="linear"):
        I.load(_write(tmp_path, "bad.toml", text.replace('"linear"', '"exponential"')))


def test_linear_schedule_matches_reference_formula():
    from mjolnir_b200.anneal import current
    assert current(350.0, 280.0, 0.0) == 350.0 and current(350.0, 280.0, 1.0) == 280.0
    assert current(300.0, 100.0, 0.25) == 300.0 * 0.75 + 100.0 * 0.25


@pytest.mark.parametrize("kind", ["WCA", "LennardJonesAttractive", "UniformLennardJones"])
def test_lj_family_round_trip(kind, tmp_path):
    from lj_family import fluid
    d = fluid(kind, n=64)
    path = str(tmp_path / "f.toml")
    I.dump(d, path)
    g = I.load(path).desc
    assert g.lj.kind == kind and g.lj.cutoff == d.lj.cutoff
    np.testing.assert_array_equal(g.lj.idx, d.lj.idx)
    np.testing.assert_array_equal(g.lj.param0, d.lj.param0)
    np.testing.assert_array_equal(g.lj.param1, d.lj.param1)


def test_uniform_lj_without_parameters_takes_every_particle(tmp_path):
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF
    start = text.index("[[forcefields.global]]")
    text = text[:start] + """[[forcefields.global]]
interaction = "Pair"
potential   = "UniformLennardJones"
sigma = 1.5
epsilon = 0.4
spatial_partition = {type = "CellList", margin = 0.3}
"""
    d = I.load(_write(tmp_path, "u.toml", text)).desc
    np.testing.assert_array_equal(d.lj.idx, np.arange(4))
    assert set(d.lj.param0) == {1.5} and set(d.lj.param1) == {0.4} and d.lj.cutoff == 2.5


@pytest.mark.parametrize("case", ["InversePower12", "InversePower6", "HardCoreExcludedVolume"])
def test_exv_family_round_trip(case, tmp_path):
    from exv_family import system
    d = system(case)
    path = str(tmp_path / "f.toml")
    I.dump(d, path)
    g = I.load(path).desc
    assert g.exv.kind == d.exv.kind and g.exv.cutoff == d.exv.cutoff and g.exv.epsilon == d.exv.epsilon
    assert g.exv.exponent == d.exv.exponent
    np.testing.assert_array_equal(g.exv.param0, d.exv.param0)
    if d.exv.param1 is not None:
        np.testing.assert_array_equal(g.exv.param1, d.exv.param1)


def test_inverse_power_default_cutoff_uses_integer_quotient(tmp_path):
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF
    start = text.index("[[forcefields.global]]")
    text = text[:start] + """[[forcefields.global]]
interaction = "Pair"
potential   = "InversePower"
epsilon = 0.5
n = 5
spatial_partition = {type = "CellList", margin = 0.3}
parameters = [{index = 0, radius = 1.0}, {index = 1, radius = 1.0}]
"""
    d = I.load(_write(tmp_path, "ip.toml", text)).desc
    assert d.exv.kind == "InversePower" and d.exv.exponent == 5 and d.exv.cutoff == 4.0   # 2^(12 // 5)


@pytest.mark.parametrize("integrator", ["UnderdampedLangevin", "G-JFLangevin", "g-BAOABLangevin", "VelocityVerlet"])
def test_integrator_round_trip(integrator, tmp_path):
    """Every supported integrator type is written and read back with its
    per-particle parameters (gammas, or the G-JF alphas)."""
    d = S.polymer_melt(nchains=2, nbeads=10, radius=30.0, seed=6)
    d.integrator = integrator
    d.gamma = np.random.default_rng(1).uniform(0.1, 2.0, d.n) if integrator != "VelocityVerlet" else np.zeros(d.n)
    path = str(tmp_path / "i.toml")
    I.dump(d, path)
    text = open(path).read()
    assert ("alphas" in text) == (integrator == "G-JFLangevin")
    g = I.load(path).desc
    assert g.integrator == integrator
    np.testing.assert_array_equal(g.gamma, d.gamma)


def test_gjf_rejects_gammas(tmp_path):
    d = S.polymer_melt(nchains=2, nbeads=10, radius=30.0, seed=6)
    d.integrator = "G-JFLangevin"
    path = str(tmp_path / "i.toml")
    I.dump(d, path)
    text = open(path).read().replace("integrator.alphas", "integrator.gammas")
    open(path, "w").write(text)
    with pytest.raises(I.InputError, match="gammas"):
        I.load(path)


def test_names_groups_attributes_and_formats(tmp_path):
    """Particle names and groups, the attributes as given and the output
    formats reach the Input, and a checkpoint written with them carries the
    names and groups the reference's saver would."""
    from mjolnir_b200 import checkpoint as K
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF
    text = text.replace('output.format = "xyz"', 'output.format = ["xyz", "dcd", "trr"]')
    inp = I.load(_write(tmp_path, "named.toml", text))
    assert inp.names == ["X", "X", "X", "C"] and inp.groups == ["NONE"] * 4
    assert inp.attributes == {"temperature": 300.0}
    assert inp.output_formats == ["xyz", "dcd", "trr"]
    assert inp.file_prefix.endswith("/" + inp.output_prefix)
    d = inp.desc
    path = str(tmp_path / "n_system.msg")
    K.write_system(path, d.pos, d.vel, np.zeros_like(d.pos), d.mass, d.periodic, d.lower, d.upper,
                   inp.attributes, inp.names, inp.groups)
    back = K.read_system(path)
    assert back["names"] == inp.names and back["groups"] == inp.groups
    assert back["attributes"] == {"temperature": 300.0}


def test_unknown_output_format_is_rejected(tmp_path):
    text = HEAD.format(path=str(tmp_path) + "/") + SIM + SYSTEM + FF
    text = text.replace('output.format = "xyz"', 'output.format = "pdb"')
    with pytest.raises(I.InputError, match="pdb"):
        I.load(_write(tmp_path, "bad_fmt.toml", text))
