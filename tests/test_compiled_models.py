"""The compiled humanoid, arm and bin models against values derived here
without the model compiler (the quadruped has its own file,
test_compiled_quadruped.py).

The oracle steps the compiler's model dump, so a wrong mass, COM, inertia,
invweight or mixed contact parameter would reach both sides of every parity
test of the mixed (humanoid / arm) and bin workloads.  Here each body's mass
properties are recomputed from the MJCF text alone (parsed with
ElementTree, not by the compiler): every geom is a uniform solid (sphere,
capsule, box, ellipsoid, or the convex hull of a mesh's vertices from
scipy) with its mass given or density x volume, placed by pos / quat /
fromto, and the geoms of a body are combined with the parallel-axis
theorem.  meaninertia and the invweights are recomputed from the FP64
oracle's own kinematics and CRBA at qpos0, and the pairs' mixed friction
from the geoms' friction attributes.
"""
import ctypes as C
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import mjb200
import oracle

DENSITY = 1000.0


def quat_mat(q):
    w, x, y, z = np.asarray(q, float) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def nums(s):
    return np.array([float(v) for v in s.split()])


def hull_solid(verts):
    """Volume, centroid and inertia tensor per unit density (about the
    centroid) of the convex hull of verts, by tetrahedra from an interior
    point (divergence form of the second moments)."""
    from scipy.spatial import ConvexHull

    h = ConvexHull(verts)
    o = verts[h.vertices].mean(axis=0)
    vol, first, second = 0.0, np.zeros(3), np.zeros((3, 3))
    for simplex, eq in zip(h.simplices, h.equations):
        a, b, c = (verts[i] - o for i in simplex)
        if np.dot(np.cross(b - a, c - a), eq[:3]) < 0:
            b, c = c, b
        det = np.dot(a, np.cross(b, c))
        vol += det / 6
        s = a + b + c
        first += det / 24 * s
        second += det / 120 * (np.outer(a, a) + np.outer(b, b) + np.outer(c, c) + np.outer(s, s))
    com = first / vol                                   # relative to o
    cov = second - vol * np.outer(com, com)             # about the centroid
    inertia = np.trace(cov) * np.eye(3) - cov
    return vol, o + com, inertia / vol                  # inertia per unit mass


def geom_solid(g, meshes):
    """(mass, COM in the body frame, inertia tensor about the COM in the
    body frame) of one geom element."""
    t = g.get("type", "sphere")
    size = nums(g.get("size", "0"))
    R = quat_mat(nums(g.get("quat"))) if g.get("quat") else np.eye(3)
    pos = nums(g.get("pos")) if g.get("pos") else np.zeros(3)
    if g.get("fromto"):
        ft = nums(g.get("fromto"))
        p0, p1 = ft[:3], ft[3:]
        pos = (p0 + p1) / 2
        axis = (p1 - p0) / np.linalg.norm(p1 - p0)
        half = np.linalg.norm(p1 - p0) / 2
    else:
        axis = R[:, 2]
        half = size[1] if len(size) > 1 else 0.0
    if t == "sphere":
        r = size[0]
        vol = 4 / 3 * np.pi * r ** 3
        unit = np.eye(3) * 0.4 * r * r
    elif t == "capsule":
        r = size[0]
        vc, vs = np.pi * r * r * 2 * half, 4 / 3 * np.pi * r ** 3
        vol = vc + vs
        i_ax = (vc * r * r / 2 + vs * 0.4 * r * r) / vol
        i_perp = (vc * (r * r / 4 + (2 * half) ** 2 / 12) + vs * (0.4 * r * r + half * half + 0.75 * half * r)) / vol
        unit = i_perp * (np.eye(3) - np.outer(axis, axis)) + i_ax * np.outer(axis, axis)
    elif t == "box":
        a, b, c = size
        vol = 8 * a * b * c
        unit = R @ np.diag([(b * b + c * c) / 3, (a * a + c * c) / 3, (a * a + b * b) / 3]) @ R.T
    elif t == "ellipsoid":
        a, b, c = size
        vol = 4 / 3 * np.pi * a * b * c
        unit = R @ np.diag([(b * b + c * c) / 5, (a * a + c * c) / 5, (a * a + b * b) / 5]) @ R.T
    elif t == "mesh":
        vol, centre, unit0 = hull_solid(meshes[g.get("mesh")])
        pos = pos + R @ centre
        unit = R @ unit0 @ R.T
    else:
        raise AssertionError(f"no solid for geom type {t}")
    mass = float(g.get("mass")) if g.get("mass") else DENSITY * vol
    return mass, pos, mass * unit


def xml_bodies(xml):
    """Mass, COM and inertia tensor (about the COM, body frame) of every
    body with geoms, in document order (= body id order, world first)."""
    root = ET.fromstring(xml)
    meshes = {m.get("name"): nums(m.get("vertex")).reshape(-1, 3) for m in root.iter("mesh")}
    out = []

    def visit(b):
        parts = [geom_solid(g, meshes) for g in b.findall("geom")]
        M = sum(p[0] for p in parts)
        com = sum(p[0] * p[1] for p in parts) / M
        I = np.zeros((3, 3))
        for m, c, Ig in parts:
            d = c - com
            I += Ig + m * (np.dot(d, d) * np.eye(3) - np.outer(d, d))
        out.append((b.get("name"), M, com, I))
        for child in b.findall("body"):
            visit(child)

    for b in root.find("worldbody").findall("body"):
        visit(b)
    return out


def body_tensor(d, b):
    R = quat_mat(d["body_iquat"].reshape(-1, 4)[b])
    return R @ np.diag(d["body_inertia"].reshape(-1, 3)[b]) @ R.T, d["body_ipos"].reshape(-1, 3)[b]


MODELS = {
    "humanoid": lambda: mjb200.models.humanoid_xml(),
    "arm": lambda: mjb200.models.arm_xml(),
    "bin64": lambda: mjb200.models.bin_xml(64, 1.0, seed=1, condim=6, cone="elliptic"),
}


@pytest.fixture(scope="module", params=sorted(MODELS))
def model_xml(request):
    xml = MODELS[request.param]()
    return request.param, xml, mjb200.load_model_from_string(xml).dump()


def test_masses_coms_and_inertias_from_the_mjcf(model_xml):
    name, xml, d = model_xml
    bodies = xml_bodies(xml)
    assert len(bodies) == int(d["sizes"][3]) - 1
    for b, (bname, M, com, I) in enumerate(bodies, start=1):
        It, ct = body_tensor(d, b)
        assert d["body_mass"][b] == pytest.approx(M, rel=1e-6), (name, bname)
        np.testing.assert_allclose(ct, com, atol=1e-6, err_msg=f"{name} {bname}")
        np.testing.assert_allclose(It, I, rtol=1e-5, atol=1e-7 * max(1.0, np.abs(I).max()), err_msg=f"{name} {bname}")


def test_meaninertia_and_invweights_from_the_oracle(model_xml):
    name, xml, d = model_xml
    om = oracle.OracleModel(d)
    env = oracle.OracleEnv(om, 64, 256)
    env.a["qpos"][:] = d["qpos0"]
    env.a["qvel"][:] = 0
    oracle.lib.oracle_kinematics(C.byref(om.c), C.byref(env.d))
    oracle.lib.oracle_com(C.byref(om.c), C.byref(env.d), None)
    oracle.lib.oracle_crb(C.byref(om.c), C.byref(env.d), None)
    nv, nb = om.nv, om.nbody
    M = env.a["M"].reshape(nv, nv)
    Minv = np.linalg.inv(M)
    assert d["opt_real"][7] == pytest.approx(np.trace(M) / nv, rel=1e-9)
    dv = np.diag(Minv).copy()
    want = dv.copy()
    for j, t in enumerate(d["jnt_type"]):
        a = d["jnt_dofadr"][j]
        if t == 0:                       # free: translation and rotation averaged
            want[a:a + 3] = dv[a:a + 3].mean()
            want[a + 3:a + 6] = dv[a + 3:a + 6].mean()
        elif t == 1:                     # ball
            want[a:a + 3] = dv[a:a + 3].mean()
    np.testing.assert_allclose(d["dof_invweight0"], want, rtol=1e-9)
    cdof = env.a["cdof"].reshape(nv, 6)
    scom = env.a["subtree_com"].reshape(nb, 3)
    xipos = env.a["xipos"].reshape(nb, 3)
    root, dofb, sub = d["body_rootid"], d["dof_bodyid"], d["body_subtreesize"]
    biw = d["body_invweight0"].reshape(nb, 2)
    for b in range(1, nb):
        off = xipos[b] - scom[root[b]]
        J = np.zeros((6, nv))
        for i in range(nv):
            if dofb[i] <= b < dofb[i] + sub[dofb[i]]:
                ang, lin = cdof[i, :3], cdof[i, 3:]
                J[:3, i] = lin + np.cross(ang, off)
                J[3:, i] = ang
        A = np.diag(J @ Minv @ J.T)
        assert biw[b, 0] == pytest.approx(A[:3].mean(), rel=1e-9, abs=1e-12), (name, b)
        assert biw[b, 1] == pytest.approx(A[3:].mean(), rel=1e-9, abs=1e-12), (name, b)
    pr = d["pair_real"].reshape(-1, 16)
    pi = d["pair_int"].reshape(-1, 6)
    np.testing.assert_allclose(pr[:, 14], biw[pi[:, 2], 0] + biw[pi[:, 3], 0], rtol=1e-12)
    np.testing.assert_allclose(pr[:, 15], biw[pi[:, 2], 1] + biw[pi[:, 3], 1], rtol=1e-12)


def test_mixed_friction_is_the_geoms_maximum(model_xml):
    """Every pair's friction is the element-wise maximum of its two geoms'
    friction attributes (defaults from the MJCF's <default> and MuJoCo's
    1 / 0.005 / 0.0001), expanded to (slide, slide, spin, roll, roll)."""
    name, xml, d = model_xml
    root = ET.fromstring(xml)
    dflt = root.find("default/geom")
    base = nums(dflt.get("friction")) if dflt is not None and dflt.get("friction") else np.array([1.0, 0.005, 0.0001])
    geoms = list(root.find("worldbody").iter("geom"))
    fr = [nums(g.get("friction")) if g.get("friction") else base for g in geoms]
    assert len(geoms) == int(d["sizes"][5])
    pr = d["pair_real"].reshape(-1, 16)
    pi = d["pair_int"].reshape(-1, 6)
    assert len(pi) > 0
    for (g1, g2), f in zip(pi[:, :2], pr[:, 2:7]):
        mx = np.maximum(fr[g1], fr[g2])
        np.testing.assert_allclose(f, [mx[0], mx[0], mx[1], mx[2], mx[2]], rtol=1e-12, err_msg=f"{name} pair {g1} {g2}")


def test_pair_table_matches_filter_rules(model_xml):
    """The candidate pairs against the filter restatement of test_model.py,
    with the geoms' contype / conaffinity read from the MJCF (default 1 / 1)
    rather than taken from the compiler."""
    from test_model import expected_pairs

    name, xml, d = model_xml
    geoms = list(ET.fromstring(xml).find("worldbody").iter("geom"))
    np.testing.assert_array_equal(d["geom_contype"], [int(g.get("contype", 1)) for g in geoms])
    np.testing.assert_array_equal(d["geom_conaffinity"], [int(g.get("conaffinity", 1)) for g in geoms])
    pi = d["pair_int"].reshape(-1, 6)
    got = {frozenset((int(a), int(b))) for a, b in pi[:, :2]}
    assert len(got) == len(pi)
    assert got == expected_pairs(d, True)


GEOM_TYPE = {"plane": 0, "hfield": 1, "sphere": 2, "capsule": 3, "ellipsoid": 4, "cylinder": 5, "box": 6, "mesh": 7}
JOINT_TYPE = {"free": 0, "ball": 1, "slide": 2, "hinge": 3}


@pytest.mark.parametrize("name", ["quadruped", "humanoid", "arm", "bin64"])
def test_kinematic_tree_from_the_mjcf(name):
    """Body frames, parents, joints and geom placement in the dump against
    the MJCF text: body pos / quat relative to the parent, joint type, pos,
    unit axis, range and armature, geom type, body, size, and for fromto
    capsules the midpoint, the half-length and the z axis along the segment
    (the oracle's kinematics reads all of these from the dump)."""
    xml = mjb200.models.quadruped_xml() if name == "quadruped" else MODELS[name]()
    d = mjb200.load_model_from_string(xml).dump()
    wb = ET.fromstring(xml).find("worldbody")
    bodies, parents = [wb], [-1]

    def visit(b, parent):
        bodies.append(b)
        parents.append(parent)
        me = len(bodies) - 1
        for c in b.findall("body"):
            visit(c, me)

    for b in wb.findall("body"):
        visit(b, 0)
    nb = int(d["sizes"][3])
    assert len(bodies) == nb
    np.testing.assert_array_equal(d["body_parentid"][1:], parents[1:])
    bpos, bquat = d["body_pos"].reshape(nb, 3), d["body_quat"].reshape(nb, 4)
    joints, geoms = [], []
    for i, b in enumerate(bodies):
        if i:
            np.testing.assert_allclose(bpos[i], nums(b.get("pos", "0 0 0")), atol=1e-12, err_msg=f"{name} body {i}")
            q = nums(b.get("quat", "1 0 0 0"))
            q /= np.linalg.norm(q)
            assert min(np.abs(bquat[i] - q).max(), np.abs(bquat[i] + q).max()) < 1e-9, (name, i)
        for el in b:
            if el.tag in ("joint", "freejoint"):
                joints.append((i, el))
            elif el.tag == "geom":
                geoms.append((i, el))
    nj = int(d["sizes"][4])
    assert len(joints) == nj
    jpos, jaxis, jrng = d["jnt_pos"].reshape(nj, 3), d["jnt_axis"].reshape(nj, 3), d["jnt_range"].reshape(nj, 2)
    for j, (bi, el) in enumerate(joints):
        t = "free" if el.tag == "freejoint" else el.get("type", "hinge")
        assert d["jnt_type"][j] == JOINT_TYPE[t] and d["jnt_bodyid"][j] == bi, (name, j)
        if t in ("hinge", "slide"):
            ax = nums(el.get("axis", "0 0 1"))
            np.testing.assert_allclose(jaxis[j], ax / np.linalg.norm(ax), atol=1e-12, err_msg=f"{name} joint {j}")
            np.testing.assert_allclose(jpos[j], nums(el.get("pos", "0 0 0")), atol=1e-12, err_msg=f"{name} joint {j}")
            if el.get("range"):
                np.testing.assert_allclose(jrng[j], nums(el.get("range")), atol=1e-12)
                assert d["jnt_limited"][j] == 1
            if el.get("armature"):
                assert d["dof_armature"][d["jnt_dofadr"][j]] == pytest.approx(float(el.get("armature")))
    ng = int(d["sizes"][5])
    assert len(geoms) == ng
    gpos, gquat, gsize = d["geom_pos"].reshape(ng, 3), d["geom_quat"].reshape(ng, 4), d["geom_size"].reshape(ng, 3)
    for g, (bi, el) in enumerate(geoms):
        t = el.get("type", "sphere")
        assert d["geom_type"][g] == GEOM_TYPE[t] and d["geom_bodyid"][g] == bi, (name, g)
        if el.get("fromto"):
            ft = nums(el.get("fromto"))
            seg = ft[3:] - ft[:3]
            np.testing.assert_allclose(gpos[g], (ft[:3] + ft[3:]) / 2, atol=1e-12)
            assert gsize[g, 0] == pytest.approx(nums(el.get("size"))[0]) and gsize[g, 1] == pytest.approx(np.linalg.norm(seg) / 2)
            np.testing.assert_allclose(quat_mat(gquat[g])[:, 2], seg / np.linalg.norm(seg), atol=1e-9)
        elif t in ("sphere", "box", "ellipsoid", "capsule", "cylinder"):
            sz = nums(el.get("size"))
            np.testing.assert_allclose(gsize[g, :len(sz)], sz, atol=1e-12)
            np.testing.assert_allclose(gpos[g], nums(el.get("pos", "0 0 0")), atol=1e-12)
