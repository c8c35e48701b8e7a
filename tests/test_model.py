"""Model compiler (MJCF -> Model) on the CPU: sizes, the collision pair table
against an independent restatement of the filter rules of the reference's
Model::init_cache (io.cpp:961-1070), contact-parameter mixing
(io.cpp:922-959, 1006-1013) and error behaviour of the loader."""
import numpy as np
import pytest

import mjb200

PLANE = '<geom type="plane" size="5 5 0.1"/>'


def test_quadruped_sizes(quad_model):
    d = quad_model.dump()
    assert (quad_model.nq, quad_model.nv, quad_model.nu) == (19, 18, 12)
    nq, nv, nu, nbody, njnt, ngeom, nmesh, npair = [int(x) for x in d["sizes"][:8]]
    assert (nbody, njnt, ngeom, nmesh) == (14, 13, 14, 0)
    assert npair == 79
    # nominal standing pose sits inside every joint range
    rng = d["jnt_range"].reshape(-1, 2)
    q0 = d["qpos0"]
    for j in range(1, njnt):
        a = d["jnt_qposadr"][j]
        assert rng[j, 0] <= mjb200.models.QUAD_NOMINAL[(j - 1) % 3] <= rng[j, 1]
        assert q0[a] == 0.0


def expected_pairs(d, self_collision=True):
    """Independent restatement of the candidate-pair filter: different weld
    bodies, not parent and child (unless the parent is the world), contype /
    conaffinity compatible, and (self_collision off) not within one tree."""
    ngeom = int(d["sizes"][5])
    body = d["geom_bodyid"]
    weld = d["body_weldid"]
    parent = d["body_parentid"]
    root = d["body_rootid"]
    ct, ca = d["geom_contype"], d["geom_conaffinity"]
    out = set()
    for g1 in range(ngeom):
        for g2 in range(g1 + 1, ngeom):
            w1, w2 = weld[body[g1]], weld[body[g2]]
            if w1 == w2:
                continue
            if w1 != 0 and w2 != 0 and (weld[parent[w1]] == w2 or weld[parent[w2]] == w1):
                continue
            if not ((ct[g1] & ca[g2]) or (ct[g2] & ca[g1])):
                continue
            if not self_collision and root[w1] == root[w2] and root[w1] != 0:
                continue
            out.add(frozenset((g1, g2)))
    return out


@pytest.mark.parametrize("self_collision", [1, 0])
def test_pair_table_matches_filter_rules(quad_xml, self_collision):
    m = mjb200.load_model_from_string(quad_xml, self_collision=self_collision)
    d = m.dump()
    pi = d["pair_int"].reshape(-1, 6)
    got = {frozenset((int(a), int(b))) for a, b in pi[:, :2]}
    assert len(got) == len(pi)  # no duplicates
    assert got == expected_pairs(d, bool(self_collision))
    gt = d["geom_type"]
    for g1, g2, b1, b2, condim, explicit in pi:
        assert gt[g1] <= gt[g2]  # type-ordered
        assert d["geom_bodyid"][g1] == b1 and d["geom_bodyid"][g2] == b2
        assert condim == max(d["geom_condim"][g1], d["geom_condim"][g2])
        assert explicit == 0


def test_pair_parameter_mixing():
    xml = ('<mujoco><worldbody>' + '<geom type="plane" size="5 5 0.1" friction="0.5 0.01 0.002" margin="0.01" gap="0.002" condim="1"/>'
           '<body pos="0 0 1"><freejoint/><geom type="sphere" size="0.1" friction="1.2 0.005 0.0001" margin="0.02" gap="0.001" condim="3"/>'
           '</body></worldbody></mujoco>')
    d = mjb200.load_model_from_string(xml).dump()
    pi = d["pair_int"].reshape(-1, 6)
    pr = d["pair_real"].reshape(-1, 16)
    assert len(pi) == 1 and pi[0, 4] == 3
    margin, gap = pr[0, 0], pr[0, 1]
    assert margin == pytest.approx(0.02) and gap == pytest.approx(0.002)
    # friction: element-wise maximum, expanded to 5 (slide, slide, spin, roll, roll)
    np.testing.assert_allclose(pr[0, 2:7], [1.2, 1.2, 0.01, 0.002, 0.002], rtol=1e-12)


def test_default_classes_and_names(quad_model):
    d = quad_model.dump()
    # position actuators: gain kp, bias (0, -kp, -kv)
    gp = d["actuator_gainprm"].reshape(-1, 3)
    bp = d["actuator_biasprm"].reshape(-1, 3)
    np.testing.assert_allclose(gp[:, 0], 20.0)
    np.testing.assert_allclose(bp, np.tile([0.0, -20.0, -0.5], (12, 1)))
    assert quad_model.name2id(1, "trunk") == 1  # mjOBJ_BODY


@pytest.mark.parametrize("xml", [
    "<mujoco><worldbody><body><geom type='sphere' size='0.1'/></worldbody></mujoco>",  # unbalanced tag
    "<mujoco><worldbody><geom type='teapot' size='0.1'/></worldbody></mujoco>",          # unknown geom type
    "not xml at all",
])
def test_bad_xml_fails_with_message(xml):
    with pytest.raises(RuntimeError) as e:
        mjb200.load_model_from_string(xml)
    assert str(e.value)


def test_dump_roundtrip_sizes(quad_model):
    d = quad_model.dump()
    nq, nv, nu, nbody, njnt, ngeom = [int(x) for x in d["sizes"][:6]]
    assert d["qpos0"].size == nq and d["dof_armature"].size == nv
    assert d["body_mass"].size == nbody and d["jnt_type"].size == njnt and d["geom_type"].size == ngeom
    assert d["body_mass"][1:].sum() == pytest.approx(6.0 + 4 * (3 * 0.7) + 4 * 0.0, rel=0.2)


def test_committed_oracle_dump_matches_compiler(quad_model):
    """The bench's CPU arm steps oracle/models/quadruped12.dump (so it never
    loads the product library); the committed dump must be what the
    compiler produces today (regenerate with oracle/make_model_dumps.py)."""
    import oracle

    want = quad_model.dump()
    got = oracle.load_dump("quadruped12.dump")
    assert sorted(got) == sorted(want)
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
