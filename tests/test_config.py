"""inp.json → cs3d_params on the CPU: every field the reader fills agrees
with the same parameters given directly, for the benchmark configurations
and with the Langevin force and the CoM correction switched on; comments in
the reference's two styles are accepted; keys of features outside the
library are refused (src/GPUbounce.cu:1914-2247 is the reference's reader)."""
import json

import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import workloads as W

# stiffness1 and stiffness2 are products of floats read from inp.json
# (stiffFactor1 x Youngs_mod, softStiffFactor x Youngs_mod, as the reference
# computes them), so they may differ from the direct value by rounding
PRODUCTS = ("stiffness1", "stiffness2")


def _direct(p, steps, seed):
    """The parameters that W.inp_json(p, ..., steps, ..., seed=seed) states:
    p, with the step count, the seed (RANMAR seeds from cs3d_seed_map) and the
    values the file carries for switched-off features (rand_scale_factor 0.1,
    softStiffFactor 1, phase_count 2e9)."""
    q = dict(p, div_time_steps=steps, rand_seed=seed)
    q["rng_ij"], q["rng_kl"] = cs.seed_map(seed)
    q.setdefault("rand_scale_factor", 0.1)
    q.setdefault("stiffness2", float(np.float32(p.get("soft_stiff_factor", 1.0)) * np.float32(p["youngs_mod"])))
    q.setdefault("phase_count", 2000000000)
    return cs.make_params(q)


def _from_json(tmp_path, d, text_edit=None, name="inp.json"):
    text = json.dumps(d, indent=1)
    if text_edit:
        text = text_edit(text)
    path = tmp_path / name
    path.write_text(text)
    return cs.config_to_params(cs.read_json_params(str(path)))


def _compare(got, want):
    for name, _t in cs.Params._fields_:
        a, b = getattr(got, name), getattr(want, name)
        if name == "box_len":
            assert list(a) == list(b), name
        elif name in PRODUCTS:
            assert np.isclose(np.float32(a), np.float32(b), rtol=2 ** -22, atol=0), (name, a, b)
        else:
            assert a == b, (name, a, b)


def _configs():
    out = [("config1", W.config1()[0]), ("config2", W.config2()[0]), ("config3", W.config3(1000)[0])]
    out += [("config4 inst %d" % k, W.config4()[k][0]) for k in (0, 17, 255)]
    out += [("config5 inst %d" % k, W.config5(n_inst=2)[k][0]) for k in (0, 1)]
    return out


@pytest.mark.parametrize("name,p", _configs(), ids=[n for n, _ in _configs()])
def test_every_field_matches_the_direct_parameters(tmp_path, name, p):
    got = _from_json(tmp_path, W.inp_json(p, 256, 1200, 100, seed=77))
    _compare(got, _direct(p, 1200, 77))


def test_langevin_and_com_correction_keys(tmp_path):
    p = W.config1()[0]
    d = W.inp_json(p, 64, 500, 10, seed=9)
    d["rand_params"].update(add_rands=True, rand_scale_factor=0.05)
    d["core"]["correct_com"] = True
    got = _from_json(tmp_path, d)
    want = _direct(dict(p, add_rands=1, rand_scale_factor=0.05, correct_com=1), 500, 9)
    _compare(got, want)


def test_comments_in_both_styles(tmp_path):
    p = W.config1()[0]
    d = W.inp_json(p, 64, 500, 10, seed=9)

    def commented(text):
        lines = text.split("\n")
        lines.insert(1, "  // line comment before the first section")
        lines.insert(3, "  /* block comment\n     over two lines */")
        return "\n".join(lines)

    _compare(_from_json(tmp_path, d, commented), _direct(p, 500, 9))


@pytest.mark.parametrize("edits", [
    {("population", "doPopModel"): 1},
    {("walls", "useWalls"): 1, ("boxParams", "useRigidSimulationBox"): False},
    {("boxParams", "usePBCs"): True},
    {("core", "doAdaptive_dt"): True},
    {("divParams", "useDivPlaneBasis"): 1},
], ids=["population model", "walls", "periodic box", "adaptive dt", "division plane basis"])
def test_features_outside_the_library_are_refused(tmp_path, edits):
    d = W.inp_json(W.config1()[0], 64, 500, 10)
    for (section, key), value in edits.items():
        d[section][key] = value
    with pytest.raises(cs.CS3DError) as e:
        _from_json(tmp_path, d)
    assert e.value.status == -8   # CS3D_E_UNSUPPORTED


def test_walls_with_a_rigid_box_fail_the_reference_validation(tmp_path):
    # the reference's own check, src/GPUbounce.cu:2234-2238: walls and a rigid box exclude each other
    d = W.inp_json(W.config1()[0], 64, 500, 10)
    d["walls"]["useWalls"] = 1
    with pytest.raises(cs.CS3DError) as e:
        _from_json(tmp_path, d)
    assert e.value.status == -6   # CS3D_E_CONFIG


def test_malformed_file_reports_a_parse_error(tmp_path):
    path = tmp_path / "bad.json"
    path.write_text('{"core": {"particle_mass": 0.04,, }')
    with pytest.raises(cs.CS3DError) as e:
        cs.read_json_params(str(path))
    assert e.value.status == -5   # CS3D_E_PARSE
