"""The .dsml loader (dem_dsml_*): against the reference's own parser and
block generators built for the host (oracle/_ref, where the reference tree
was present at build time), on the reference's example scenes and on a test
scene of every block kind; the reference's error messages; its grid rule;
the seeded jitter."""
import glob
import math
import os

import numpy as np
import pytest

from demso_b200 import dsml, scenes
from demso_b200._lib import DemError
from oracle.oracle import RefDsml, dsml_ref_available, ref_root

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "dsml", "blocks.dsml")
# the reference's example scenes, where its checkout is present ($REF_ROOT)
EXAMPLES = sorted(glob.glob(os.path.join(ref_root(), "exemplos", "*.dsml"))) if ref_root() else []
need_ref = pytest.mark.skipif(not dsml_ref_available(), reason="reference host build absent")


def compare_with_reference(path, tmp_path):
    ref = RefDsml().load(path, str(tmp_path))
    if "error" in ref:
        with pytest.raises(DemError) as e:
            dsml.load(path)
        assert ref["error"] in str(e.value)
        return None
    s = dsml.load(path, jitter=False)
    ts, dur, img, lx, ly, gx, gy, kn, kt = ref["params"]
    assert (np.float32(ts), np.float32(dur), int(img)) == (s.time_step, s.sim_duration,
                                                           s.image_height)
    sy = s.system
    assert (np.float32(lx), np.float32(ly)) == (np.float32(sy.Lx), np.float32(sy.Ly))
    assert (np.float32(gx), np.float32(gy)) == (np.float32(sy.gravity[0]),
                                                np.float32(sy.gravity[1]))
    assert (np.float32(kn), np.float32(kt)) == (np.float32(sy.knWall), np.float32(sy.ktWall))
    assert len(ref["types"]) == len(s.types) == len(sy.materials)
    for t, (rt, mt, mat) in enumerate(zip(ref["types"], s.types, sy.materials)):
        mass, radius, kn_, kt_, cn, eb, mu, at = rt["values"]
        assert rt["id"] == mt["id"]
        assert (np.float32(mass), np.float32(radius)) == (mt["mass"], mt["radius"])
        assert [np.float32(x) for x in (kn_, kt_, cn, eb, mu, at)] == \
            [np.float32(x) for x in mat.row()]
    assert list(s.followed) == ref["followed"]
    assert np.array_equal(s.pos, ref["pos"])
    assert np.array_equal(s.id, ref["id"]) and np.array_equal(s.type, ref["type"])
    radii = np.array([t["radius"] for t in s.types], np.float32)
    masses = np.array([t["mass"] for t in s.types], np.float32)
    assert np.array_equal(s.radius, radii[s.type]) and np.array_equal(s.mass, masses[s.type])
    return s


@need_ref
@pytest.mark.parametrize("path", EXAMPLES, ids=[os.path.basename(p) for p in EXAMPLES])
def test_reference_examples_match_the_reference_parser(path, tmp_path):
    compare_with_reference(path, tmp_path)


@need_ref
def test_block_fixture_matches_the_reference_parser(tmp_path):
    s = compare_with_reference(FIXTURE, tmp_path)
    assert s is not None


def test_block_fixture_layout():
    """Singles first (3), then the rectangles (17 x 12, 5 x 4), then the
    triangle (13 on its base: 91); ids in that order; types cycle as the
    generators cycle them; the triangle's rows hold 13, 12, ... particles."""
    s = dsml.load(FIXTURE, jitter=False)
    assert s.n == 3 + 17 * 12 + 5 * 4 + 91
    assert np.array_equal(s.id, np.arange(s.n, dtype=np.uint32))
    assert list(s.followed) == [0, 2, 7, 40]
    assert [t["id"] for t in s.types] == ["sand", "clay", "rock"]
    assert s.types[0]["name"] == "Sand & grit"
    assert s.types[0]["color"] == (0xc2, 0xb2, 0x80) and s.types[2]["color"] == (255, 255, 255)
    assert list(s.type[:3]) == [2, 0, 0]
    assert np.array_equal(s.vel[0], np.float32([-0.5, 0.1]))
    assert s.theta[0] == np.float32(0.3) and s.omega[2] == np.float32(-1.5)
    rect = s.type[3:3 + 204].reshape(12, 17)
    ij = np.add.outer(np.arange(12), np.arange(17))
    assert np.array_equal(rect, np.array([0, 1], np.uint32)[ij % 2])
    assert np.all(s.type[207:227] == 0)
    tri = s.pos[227:]
    rows = np.unique(tri[:, 1])
    assert [int(np.sum(tri[:, 1] == y)) for y in rows] == list(range(13, 0, -1))
    assert s.time_step == np.float32(5e-5) and s.sim_duration == np.float32(0.25)
    assert s.image_height == 480 and s.controlled_type == -1
    assert len(s.system.materials) == 3 and s.system.materials[1].attractCoefficient == 5.0


def test_grid_rule_is_the_reference_rule():
    """dem_dsml_system's grid against the restatement of main.cu:218-236 in
    scenes.reference_grid (float arithmetic, y measured with the x size)."""
    rng = np.random.default_rng(4)
    for _ in range(40):
        lx, ly = (float(v) for v in rng.uniform(0.05, 20.0, size=2))
        r = float(rng.uniform(0.001, 0.2))
        text = open(FIXTURE).read()
        text = text.replace("<dimensions><x>1.5</x><y>1.0</y></dimensions>",
                            "<dimensions><x>%.9g</x><y>%.9g</y></dimensions>" % (lx, ly))
        for old in ("12e-3", "15e-3", "40e-3"):
            text = text.replace("<radius>%s</radius>" % old, "<radius>%.9g</radius>" % r)
        s = dsml.parse(text)
        lx, ly, r = (float(np.float32("%.9g" % v)) for v in (lx, ly, r))
        assert (s.system.gx, s.system.gy) == scenes.reference_grid(lx, ly, r)


ERRORS = [
    ("<timestep>", "<notatimestep>", "Simulation timestep not specified"),
    ('<stiffness dir="shear">5e3', '<stiffness dir="sideways">5e3',
     "Unrecognized stiffness direction"),
    ("<friction>0.5</friction>", "<friction>0.5</friction><colour>1</colour>",
     "Unrecognized tag inside <particletype>"),
    ('particletype="clay,sand,rock"', 'particletype="clay,silt"',
     "Nonexistant particle id: 'silt'"),
    ("<start><x>0.1</x><y>0.1</y></start>", "", "<start> tag not found inside rectangle"),
    ("<width>0.5</width>", "", "<width> tag not found inside triangle"),
    ("<pos><x>0.8</x><y>0.9</y></pos>", "", "Missing <pos> tag on particle definition"),
    ('<damping type="boundary">0.4', '<damping type="wall">0.4', "Unrecognized damping type"),
]


@pytest.mark.parametrize("old,new,msg", ERRORS, ids=[e[2][:30] for e in ERRORS])
def test_parse_errors_carry_the_reference_messages(old, new, msg, tmp_path):
    text = open(FIXTURE).read()
    assert old in text
    bad = text.replace(old, new, 1).replace("</notatimestep>", "</notatimestep>")
    if old == "<timestep>":
        bad = bad.replace("</timestep>", "</notatimestep>")
    with pytest.raises(DemError) as e:
        dsml.parse(bad)
    assert msg in str(e.value)
    if dsml_ref_available():
        p = tmp_path / "bad.dsml"
        p.write_text(bad)
        assert RefDsml().load(str(p), str(tmp_path)) == {"error": msg}


def test_malformed_xml_is_an_error():
    for text in ("<simulation><parameters>", "<simulation></parameters>", "<a b=c></a>"):
        with pytest.raises(DemError):
            dsml.parse(text)


def test_rectangle_jitter_is_seeded():
    """Lattice points move by (N(0,1) - 0.5) / 100 of the spacing per axis:
    the same seed gives the same scene, another seed another one, and the
    offsets have that mean and spread."""
    a = dsml.load(FIXTURE, seed=11)
    b = dsml.load(FIXTURE, seed=11)
    c = dsml.load(FIXTURE, seed=12)
    z = dsml.load(FIXTURE, jitter=False)
    assert np.array_equal(a.pos, b.pos) and not np.array_equal(a.pos, c.pos)
    sl = slice(3, 3 + 204)
    dx = (a.pos[sl, 0].astype(np.float64) - z.pos[sl, 0]) / (0.5 / 16) * 100
    dy = (a.pos[sl, 1].astype(np.float64) - z.pos[sl, 1]) / (0.35 / 11) * 100
    d = np.concatenate([dx, dy])
    assert abs(d.mean()) < 0.2 and 0.85 < d.std() < 1.15
    # singles and triangles are not jittered
    assert np.array_equal(a.pos[:3], z.pos[:3]) and np.array_equal(a.pos[227:], z.pos[227:])
