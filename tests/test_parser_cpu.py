"""The config parser against the reference's own parser tests (tests/test_parser.cpp of the reference):
the same documents give the same error key and code, and the same defaults. The reference tests call
its section parsers one by one; here every document goes through the full parse_config, so each case
carries the sections before the failing one in a valid form."""
import copy

import numpy as np
import pytest

import sqsgenerator_b200 as S
from sqsgenerator_b200.core import ParseErrorCode as E

# test_parser.cpp:29-32: a rectangular cell with four sites (Na, Mg, Al, Si)
LATTICE = [[1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 3.0]]
COORDS = [[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]]
SPECIES = [11, 12, 13, 14]


def structure(supercell=(1, 1, 1)):
    """test_parser.cpp:34-42"""
    return {"structure": {"lattice": copy.deepcopy(LATTICE), "coords": copy.deepcopy(COORDS),
                          "species": list(SPECIES), "supercell": list(supercell)}}


def with_composition(supercell=(1, 1, 1)):
    """test_parser.cpp:44-52: Ni and Co on all sites"""
    n = supercell[0] * supercell[1] * supercell[2]
    doc = structure(supercell)
    doc["composition"] = {"Ni": 2 * n, "Co": 2 * n}
    return doc


def with_two_sublattices(supercell=(1, 1, 1)):
    """test_parser.cpp:54-62: Ni/Co on the Al and Mg sites, B/N on the rest"""
    n = supercell[0] * supercell[1] * supercell[2]
    doc = structure(supercell)
    doc["composition"] = [{"Ni": n, "Co": n, "sites": ["Al", "Mg"]}, {"B": n, "N": n}]
    return doc


def error(doc):
    res = S.parse_config(doc)
    assert isinstance(res, S.ParseError), res
    return res.key, res.code


def test_empty_document_fails():
    """test_parser.cpp:83-86"""
    assert error({}) == ("structure", E.not_found)


@pytest.mark.parametrize("species,key,codes", [
    (None, "species", {E.not_found}),                         # :113-114
    ([1, 2, 3], "species", {E.out_of_range}),                 # :115-116 wrong count
    ([1, 2, 3, -5], "species", {E.out_of_range}),             # :119-120 invalid atomic number
    (["Al", "Mg", "Si", "??"], "species", {E.out_of_range}),  # :122-124 invalid symbol
])
def test_structure_species_errors(species, key, codes):
    doc = with_composition()
    if species is None:
        del doc["structure"]["species"]
    else:
        doc["structure"]["species"] = species
    k, c = error(doc)
    assert k == key and c in codes


def test_structure_shape_errors():
    """test_parser.cpp:126-135: coords of the wrong shape; lattice and coords swapped"""
    doc = with_composition()
    doc["structure"]["species"] = ["Al", "Mg", "Si", "Ge"]
    doc["structure"]["coords"] = [1, 2, 3, 4]
    assert error(doc) == ("coords", E.type_error)
    doc["structure"]["lattice"] = copy.deepcopy(COORDS)
    doc["structure"]["coords"] = copy.deepcopy(LATTICE)
    k, c = error(doc)
    assert k == "lattice" and c in (E.out_of_range, E.type_error)


@pytest.mark.parametrize("composition,key,code", [
    ([], "composition", E.out_of_range),                        # :152-153
    ({"Ni": -1}, "composition", E.bad_value),                    # :155-160
    ([{"Ni": -1}], "composition", E.bad_value),
    ({"Ni": "1"}, "composition", E.type_error),                  # :162-167
    ([{"Ni": "1"}], "composition", E.type_error),
    ({"_Ni": "1"}, "composition", E.out_of_range),               # :169-174 invalid symbol
    ([{"_Ni": "1"}], "composition", E.out_of_range),
    ({"Ni": 3, "Fe": 2}, "sites", E.out_of_range),               # :176-181 five atoms on four sites
    ([{"Ni": 3, "Fe": 2}], "sites", E.out_of_range),
])
def test_composition_species_errors(composition, key, code):
    doc = structure()
    assert error(doc) == ("composition", E.not_found)  # :150
    doc["composition"] = composition
    assert error(doc) == (key, code)


@pytest.mark.parametrize("sites", [
    [-1, 2],           # :196-198 invalid index
    [],                # :199-201 no sites
    [0, 2],            # :203-205 two sites for four atoms
    "Fr",              # :207-209 a species the structure does not hold
    ["Si", "Mg"],      # :211-213 two sites by symbol
])
def test_composition_sites_errors(sites):
    doc = structure()
    doc["composition"] = {"Ni": 2, "Co": 2, "sites": sites}
    assert error(doc) == ("sites", E.out_of_range)


def test_composition_sites_with_invalid_species_symbol():
    """test_parser.cpp:215-217: the sites are valid, a species symbol is not"""
    doc = structure()
    doc["composition"] = {"Ni": 1, "_Co": 1, "sites": ["Si", "Mg"]}
    assert error(doc) == ("sites", E.out_of_range)


def test_split_composition_errors():
    """test_parser.cpp:220-263: overlapping sublattices (by index, by symbols, by one symbol), and a
    sublattice without sites that holds more atoms than the sites left"""
    doc = structure()
    doc["sublattice_mode"] = "split"
    sl1 = {"Ni": 1, "Co": 1, "sites": [0, 1]}
    doc["composition"] = [sl1, {"Ni": 1, "Co": 1, "sites": [1, 2]}]
    assert error(doc) == ("sites", E.bad_value)
    doc["composition"][1]["sites"] = ["Na", "Si"]
    assert error(doc) == ("sites", E.bad_value)
    doc["composition"][1]["sites"] = "Mg"
    assert error(doc) == ("sites", E.bad_value)
    del doc["composition"][1]["sites"]
    doc["composition"][1]["Ni"] = 2
    assert error(doc) == ("sites", E.out_of_range)


def _radii(doc):
    c = S.parse_config(doc)
    assert not isinstance(c, S.ParseError), c
    return [list(r) for r in c.shell_radii]


def test_shell_radii_default_and_peak():
    """test_parser.cpp:267-279"""
    doc = with_composition((2, 2, 2))
    assert _radii(doc)
    doc["shell_radii"] = "peak"
    assert _radii(doc)


def test_shell_radii_naive_equals_histogram_on_a_perfect_lattice():
    """test_parser.cpp:281-294: with a small bin width the histogram method finds the naive shells"""
    doc = with_composition((2, 2, 2))
    doc["bin_width"] = 0.001
    default = _radii(doc)
    doc["shell_radii"] = "naive"
    assert np.allclose(default, _radii(doc), rtol=0, atol=1e-9)


def test_shell_radii_naive_equals_histogram_per_sublattice():
    """test_parser.cpp:296-309"""
    doc = with_two_sublattices((2, 2, 2))
    doc["sublattice_mode"] = "split"
    doc["bin_width"] = 0.001
    default = _radii(doc)
    doc["shell_radii"] = ["naive", "naive"]
    naive = _radii(doc)
    assert len(default) == len(naive) == 2
    for a, b in zip(default, naive):
        assert np.allclose(a, b, rtol=0, atol=1e-9)


def test_shell_weights_errors():
    """test_parser.cpp:311-335: shell 0, a shell that does not exist, and one dict per sublattice in
    interact mode"""
    doc = with_composition()
    doc["shell_weights"] = {"0": 0.0}
    assert error(doc) == ("shell_weights", E.bad_value)
    doc["shell_weights"] = {"200": 200.0}
    assert error(doc) == ("shell_weights", E.out_of_range)
    doc["shell_weights"] = [{"1": 1.0, "2": 2.0}, {"1": 1.0, "2": 2.0}]
    assert error(doc) == ("shell_weights", E.bad_value)


def test_shell_weights_default():
    """test_parser.cpp:337-359: one weight set in interact mode; per sublattice in split mode, 1/k for
    every shell"""
    c = S.parse_config(with_composition((2, 2, 2)))
    assert not isinstance(c, S.ParseError), c
    assert len(c.shell_weights) == 1
    doc = with_two_sublattices((2, 2, 2))
    doc["sublattice_mode"] = "split"
    c = S.parse_config(doc)
    assert not isinstance(c, S.ParseError), c
    assert len(c.shell_weights) == 2
    want = {k: 1.0 / k for k in range(1, 9)}
    for w in c.shell_weights:
        assert dict(w) == want


def test_arrays_interact_mode_with_two_sublattices():
    """test_parser.cpp:361-370: interact mode holds one cube per array, whatever the composition"""
    c = S.parse_config(with_two_sublattices((3, 3, 3)))
    assert not isinstance(c, S.ParseError), c
    assert len(c.pair_weights) == len(c.target_objective) == len(c.prefactors) == 1


def _re_w_first():
    """The reference's "re-w.first" template: bcc Re-W 50/50, 3x3x3, first shell only, at most 10
    results per objective."""
    a = 3.165
    return {"structure": {"lattice": [[a, 0, 0], [0, a, 0], [0, 0, a]], "coords": [[0, 0, 0], [0.5, 0.5, 0.5]],
                          "species": ["W", "Re"], "supercell": [3, 3, 3]},
            "iterations": 50_000_000, "shell_weights": {"1": 1.0}, "composition": {"W": 27, "Re": 27},
            "max_results_per_objective": 10}


def _ti_al_b_n():
    """The reference's "ti-al-b-n" template: rocksalt TiN 3x3x3 in split mode, TiAl on the metal sites
    towards ordering (target -1), NB on the non-metal sites towards clustering (target +1)."""
    a = 4.253534
    coords = [[0.5, 0, 0], [0.5, 0.5, 0.5], [0, 0, 0.5], [0, 0.5, 0], [0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5],
              [0.5, 0.5, 0]]
    return {"iterations": 1_000_000_000, "sublattice_mode": "split",
            "structure": {"supercell": [3, 3, 3], "species": ["Ti"] * 4 + ["N"] * 4,
                          "lattice": [[a, 0, 0], [0, a, 0], [0, 0, a]], "coords": coords},
            "composition": [{"sites": "Ti", "Ti": 54, "Al": 54}, {"sites": "N", "N": 54, "B": 54}],
            "target_objective": [-1, 1]}


def test_templates_parse_like_the_reference():
    """The reference's shipped templates (its test_templates.py runs them through the CLI) parse, and
    carry what they say: sites, shells, caps, per-sublattice targets."""
    c = S.parse_config(_re_w_first())
    assert not isinstance(c, S.ParseError), c
    assert c.iterations == 50_000_000 and c.max_results_per_objective == 10
    assert list(c.shell_weights[0]) == [1] and len(c.composition) == 1
    assert len(c.composition[0].sites) == 54
    c = S.parse_config(_ti_al_b_n())
    assert not isinstance(c, S.ParseError), c
    assert int(c.sublattice_mode) == int(S.SublatticeMode.split) and len(c.composition) == 2
    assert [len(sl.sites) for sl in c.composition] == [108, 108]
    assert np.all(c.target_objective[0] == -1) and np.all(c.target_objective[1] == 1)


def test_templates_take_the_fast_paths():
    """Without a device, the plan of each template: the bit-mask path for the 54-site binary bcc cell,
    the lattice path for both rocksalt sublattices."""
    from sqsgenerator_b200 import _native as N
    from sqsgenerator_b200.optimize import build_job

    def plan(cfg):
        c = S.parse_config(cfg)
        d = S.prepare(c)
        job, _ = build_job(c, d)
        return N.plan(job)

    p = plan({**_re_w_first(), "iterations": 1000})
    assert [x["path"] for x in p["parts"]] == ["bitmask"] and p["shuffle_draws"] == 27
    p = plan({**_ti_al_b_n(), "iterations": 1000})
    assert [x["path"] for x in p["parts"]] == ["lattice", "lattice"] and p["shuffle_draws"] == 54 + 54
