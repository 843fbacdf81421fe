"""The benchmark configurations written in the reference's input form
(amdkiit_b200/write_inputs.py: input.yaml, input_coordinate.xyz, GTH as UPF
v2) read back through the reference-format readers (inputs.py, restating
yamlread.f90 and readupf.f90) into the same System that configs.py builds:
cell, cutoff, functional, positions and every pseudopotential array."""
import os

import numpy as np
import pytest
import yaml

from amdkiit_b200 import write_inputs
from amdkiit_b200.inputs import load_reference_input


@pytest.fixture(scope="module")
def written(tmp_path_factory):
    root = str(tmp_path_factory.mktemp("ref_inputs"))
    write_inputs.write_all(root)
    return root


@pytest.mark.parametrize("name", sorted(write_inputs.benchmark_inputs()))
def test_inputs_read_back_to_the_same_system(name, written):
    s, task, _ = write_inputs.benchmark_inputs()[name]
    r = load_reference_input(os.path.join(written, name))
    assert np.array_equal(r.a_cell, s.a_cell) and r.alat == s.alat and r.symmetry == s.symmetry
    assert r.ecut == s.ecut and r.xc == s.xc and r.nstate == s.nstate
    assert r.na == s.na and [sp.label for sp in r.species] == [sp.label for sp in s.species]
    for a, b in zip(r.positions, s.positions):
        assert np.array_equal(a, b)
    for a, b in zip(r.species, s.species):
        assert (a.z, a.zv, a.kind, a.upf_lmax, a.nbeta) == (b.z, b.zv, b.kind, b.upf_lmax, b.nbeta)
        for k in ("rr", "rab", "vloc", "beta", "dij"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), (a.label, k)
        assert list(a.beta_l) == list(b.beta_l)
    cfg = yaml.safe_load(open(os.path.join(written, name, "input.yaml")))
    assert cfg["TASK"] == task and cfg["CUTOFF"]["VALUE"] == s.ecut


def test_upf_line_layout_follows_the_reference_reader(written):
    """readupf.f90 reads line by line: the beta attributes one per line in
    its order ending with '>', PP_DIJ right after the betas (right after
    <PP_NONLOCAL> for a local-only species), and the header attributes it
    looks for."""
    for fn, nb in (("O_GTH.upf", 1), ("H_GTH.upf", 0), ("Si_GTH.upf", 2)):
        lines = open(os.path.join(written, "pseudo", fn)).read().splitlines()
        i = lines.index("<PP_NONLOCAL>")
        for k in range(nb):
            assert lines[i + 1].startswith("<PP_BETA.%d" % (k + 1))
            keys = [ln.split("=")[0] for ln in lines[i + 2:i + 10]]
            assert keys == ["type", "size", "columns", "index", "label", "angular_momentum", "cutoff_radius_index",
                            "cutoff_radius"]
            assert lines[i + 9].endswith(">")
            i = lines.index("</PP_BETA.%d>" % (k + 1))
        assert lines[i + 1].startswith("<PP_DIJ")
        head = "\n".join(lines[lines.index("<PP_HEADER"):lines.index("<PP_MESH>")])
        for key in ("element", "z_valence", "l_max", "l_local", "mesh_size", "number_of_wfc", "number_of_proj"):
            assert key + '="' in head
