"""Procedural MJCF generators for the batched-step workloads.

Each generator returns MJCF text that the library's compiler (and MuJoCo C,
where it exists) loads.  The quadruped follows the workload definition:
free-joint trunk box 0.19 x 0.05 x 0.04 m (half sizes), 6 kg; four legs of
three hinges (abduction +-0.8 rad, hip +-1.5 rad, knee -2.7..-0.9 rad) with
capsule links r = 0.02 m, length 0.213 m, 0.7 kg; spherical feet r = 0.022 m;
ground plane with friction 1.0; position actuators kp = 20, kv = 0.5; condim 3,
pyramidal cone, self-collision on; dt 0.005, Newton 16 iterations, tol 1e-8.

Choices the workload leaves open, fixed here and used everywhere:
  * abduction (hip) bodies carry an explicit 0.5 kg inertial (no geom);
  * thigh bodies sit 0.08 m outboard of the abduction axis;
  * foot spheres weigh 0.05 kg and belong to the calf body;
  * hinge armature 0.01 kg m^2, no joint damping;
  * nominal standing pose (abduction 0, hip 0.9, knee -1.8) rad, inside the
    joint ranges, so joint offsets N(0, 0.1) start near a feasible pose.
"""
from __future__ import annotations

import math

import numpy as np

QUAD_NOMINAL = (0.0, 0.9, -1.8)
QUAD_RANGES = ((-0.8, 0.8), (-1.5, 1.5), (-2.7, -0.9))
QUAD_LEGS = (("FR", 1, -1), ("FL", 1, 1), ("RR", -1, -1), ("RL", -1, 1))


def quadruped_xml(self_collision: bool = True, iterations: int = 16, tolerance: float = 1e-8,
                  timestep: float = 0.005, cone: str = "pyramidal", condim: int = 3) -> str:
    L, r, rf = 0.213, 0.02, 0.022
    con = 'contype="1" conaffinity="1"' if self_collision else 'contype="1" conaffinity="0"'
    legs = []
    for name, sx, sy in QUAD_LEGS:
        legs.append(f"""
      <body name="{name}_hip" pos="{0.19*sx:.4f} {0.05*sy:.4f} 0">
        <inertial pos="0 0 0" mass="0.5" diaginertia="0.0003 0.0003 0.0003"/>
        <joint name="{name}_abd" type="hinge" axis="1 0 0" range="{QUAD_RANGES[0][0]} {QUAD_RANGES[0][1]}" armature="0.01"/>
        <body name="{name}_thigh" pos="0 {0.08*sy:.4f} 0">
          <joint name="{name}_hipj" type="hinge" axis="0 1 0" range="{QUAD_RANGES[1][0]} {QUAD_RANGES[1][1]}" armature="0.01"/>
          <geom name="{name}_thigh_g" type="capsule" fromto="0 0 0 0 0 {-L}" size="{r}" mass="0.7" {con}/>
          <body name="{name}_calf" pos="0 0 {-L}">
            <joint name="{name}_knee" type="hinge" axis="0 1 0" range="{QUAD_RANGES[2][0]} {QUAD_RANGES[2][1]}" armature="0.01"/>
            <geom name="{name}_calf_g" type="capsule" fromto="0 0 0 0 0 {-L}" size="{r}" mass="0.7" {con}/>
            <geom name="{name}_foot" type="sphere" pos="0 0 {-L}" size="{rf}" mass="0.05" {con}/>
          </body>
        </body>
      </body>""")
    acts = []
    for name, _, _ in QUAD_LEGS:
        for j, jn in enumerate(("abd", "hipj", "knee")):
            lo, hi = QUAD_RANGES[j]
            acts.append(f'    <position name="{name}_{jn}_act" joint="{name}_{jn}" kp="20" kv="0.5" ctrlrange="{lo} {hi}"/>')
    return f"""<mujoco model="quadruped12">
  <compiler angle="radian"/>
  <option timestep="{timestep}" iterations="{iterations}" tolerance="{tolerance}" cone="{cone}" integrator="Euler"/>
  <default><geom condim="{condim}"/></default>
  <worldbody>
    <geom name="floor" type="plane" size="0 0 1" friction="1 0.005 0.0001"/>
    <body name="trunk" pos="0 0 0.3">
      <freejoint name="root"/>
      <geom name="trunk_g" type="box" size="0.19 0.05 0.04" mass="6" {con}/>{''.join(legs)}
    </body>
  </worldbody>
  <actuator>
{chr(10).join(acts)}
  </actuator>
</mujoco>
"""


def quadruped_initial_state(num_envs: int, seed0: int = 1000, env_offset: int = 0):
    """Seeded initial qpos/qvel for the quadruped (nq 19, nv 18).

    Env e uses numpy Philox(key = seed0 + e): trunk height U[0.28, 0.34],
    identity orientation, joint angles = nominal pose + N(0, 0.1) clipped into
    the joint range, zero velocity.  The host generates these once and uploads
    them, so every backend sees identical inputs.
    """
    qpos = np.zeros((num_envs, 19), np.float64)
    for i in range(num_envs):
        g = np.random.Generator(np.random.Philox(key=seed0 + env_offset + i))
        qpos[i, 2] = g.uniform(0.28, 0.34)
        qpos[i, 3] = 1.0
        off = g.normal(0.0, 0.1, size=12)
        for leg in range(4):
            for j in range(3):
                lo, hi = QUAD_RANGES[j]
                qpos[i, 7 + 3 * leg + j] = np.clip(QUAD_NOMINAL[j] + off[3 * leg + j], lo, hi)
    qvel = np.zeros((num_envs, 18), np.float64)
    return qpos, qvel


def quadruped_controls(num_envs: int, step: int, seed0: int = 2000, env_offset: int = 0):
    """Position targets U[joint range] for control step `step`, env e keyed by
    Philox(key = seed0 + e, counter = step) so any step is reproducible alone."""
    ctrl = np.zeros((num_envs, 12), np.float64)
    lo = np.array([QUAD_RANGES[j % 3][0] for j in range(12)])
    hi = np.array([QUAD_RANGES[j % 3][1] for j in range(12)])
    for i in range(num_envs):
        bitgen = np.random.Philox(key=seed0 + env_offset + i, counter=step)
        g = np.random.Generator(bitgen)
        ctrl[i] = lo + (hi - lo) * g.random(12)
    return ctrl


def quadruped_controls_fast(num_envs: int, step: int, seed: int = 2000):
    """Vectorised control draw for large batches (one Philox stream per step)."""
    g = np.random.Generator(np.random.Philox(key=seed, counter=step))
    lo = np.array([QUAD_RANGES[j % 3][0] for j in range(12)])
    hi = np.array([QUAD_RANGES[j % 3][1] for j in range(12)])
    return lo + (hi - lo) * g.random((num_envs, 12))


def quadruped_initial_state_fast(num_envs: int, seed: int = 1000):
    """Vectorised initial-state draw for large batches (same distribution as
    quadruped_initial_state, one Philox stream for the whole batch)."""
    g = np.random.Generator(np.random.Philox(key=seed))
    qpos = np.zeros((num_envs, 19), np.float64)
    qpos[:, 2] = g.uniform(0.28, 0.34, size=num_envs)
    qpos[:, 3] = 1.0
    off = g.normal(0.0, 0.1, size=(num_envs, 12))
    for leg in range(4):
        for j in range(3):
            lo, hi = QUAD_RANGES[j]
            qpos[:, 7 + 3 * leg + j] = np.clip(QUAD_NOMINAL[j] + off[:, 3 * leg + j], lo, hi)
    return qpos, np.zeros((num_envs, 18))


# ---------------------------------------------------------------- humanoid

HUMANOID_JOINTS = (
    # name, axis, range (rad)
    ("abdomen_y", "0 1 0", (-1.0, 0.5)),
    ("right_hip_x", "1 0 0", (-0.5, 0.1)), ("right_hip_z", "0 0 1", (-1.0, 0.6)), ("right_hip_y", "0 1 0", (-1.8, 0.35)),
    ("right_knee", "0 -1 0", (-2.6, -0.03)), ("right_ankle_y", "0 1 0", (-0.8, 0.8)),
    ("left_hip_x", "-1 0 0", (-0.5, 0.1)), ("left_hip_z", "0 0 -1", (-1.0, 0.6)), ("left_hip_y", "0 1 0", (-1.8, 0.35)),
    ("left_knee", "0 -1 0", (-2.6, -0.03)), ("left_ankle_y", "0 1 0", (-0.8, 0.8)),
    ("right_shoulder1", "2 1 1", (-1.5, 1.0)), ("right_shoulder2", "0 -1 1", (-1.5, 1.0)), ("right_elbow", "0 -1 1", (-1.5, 0.9)),
    ("left_shoulder1", "2 -1 1", (-1.0, 1.5)), ("left_shoulder2", "0 1 1", (-1.0, 1.5)), ("left_elbow", "0 -1 -1", (-1.5, 0.9)),
)


def humanoid_xml(iterations: int = 16, tolerance: float = 1e-8, timestep: float = 0.005) -> str:
    """21-DoF-class capsule humanoid: free-joint torso and 17 hinges (1 spine,
    2 x 5 legs, 2 x 3 arms), capsule radii 0.04-0.06 m, sphere head,
    position actuators on every hinge, self-collision on (parent/child pairs
    filtered).  nq 24, nv 23, nu 17."""
    J = {n: (a, r) for n, a, r in HUMANOID_JOINTS}

    def joint(n, pos="0 0 0"):
        a, (lo, hi) = J[n]
        return f'<joint name="{n}" type="hinge" pos="{pos}" axis="{a}" range="{lo} {hi}" armature="0.02" damping="0.5"/>'

    def leg(side, sy):
        s = side
        return f"""
          <body name="{s}_thigh" pos="0 {0.1*sy:.3f} -0.04">
            {joint(s+"_hip_x")}{joint(s+"_hip_z")}{joint(s+"_hip_y")}
            <geom name="{s}_thigh_g" type="capsule" fromto="0 0 0 0 {0.01*sy:.3f} -0.34" size="0.06"/>
            <body name="{s}_shin" pos="0 {0.01*sy:.3f} -0.403">
              {joint(s+"_knee", "0 0 .02")}
              <geom name="{s}_shin_g" type="capsule" fromto="0 0 0 0 0 -0.3" size="0.05"/>
              <body name="{s}_foot" pos="0 0 -0.39">
                {joint(s+"_ankle_y", "0 0 0.08")}
                <geom name="{s}_foot_g" type="capsule" fromto="-0.07 0 0.04 0.14 0 0.04" size="0.04"/>
              </body>
            </body>
          </body>"""

    def arm(side, sy):
        s = side
        return f"""
      <body name="{s}_upper_arm" pos="0 {0.17*sy:.3f} 0.06">
        {joint(s+"_shoulder1")}{joint(s+"_shoulder2")}
        <geom name="{s}_uarm_g" type="capsule" fromto="0 0 0 .16 {0.16*sy:.3f} -.16" size="0.04"/>
        <body name="{s}_lower_arm" pos=".18 {0.18*sy:.3f} -.18">
          {joint(s+"_elbow")}
          <geom name="{s}_larm_g" type="capsule" fromto="0.01 {0.01*sy:.3f} 0.01 .17 {0.17*sy:.3f} .17" size="0.04"/>
        </body>
      </body>"""

    acts = []
    for n, _, (lo, hi) in HUMANOID_JOINTS:
        kp = 40 if ("shoulder" in n or "elbow" in n) else 100
        acts.append(f'    <position name="{n}_act" joint="{n}" kp="{kp}" kv="2" ctrlrange="{lo} {hi}"/>')
    return f"""<mujoco model="humanoid21">
  <compiler angle="radian"/>
  <option timestep="{timestep}" iterations="{iterations}" tolerance="{tolerance}" cone="pyramidal" integrator="Euler"/>
  <default><geom condim="3" density="1000" friction="0.9 0.005 0.0001"/></default>
  <worldbody>
    <geom name="floor" type="plane" size="0 0 1" friction="1 0.005 0.0001"/>
    <body name="torso" pos="0 0 1.3">
      <freejoint name="root"/>
      <geom name="torso_g" type="capsule" fromto="0 -.07 0 0 .07 0" size="0.06"/>
      <geom name="head" type="sphere" pos="0 0 .19" size=".09"/>
      <geom name="uwaist" type="capsule" fromto="-.01 -.06 -.12 -.01 .06 -.12" size="0.05"/>
      <body name="lower_waist" pos="-.01 0 -.26">
        <geom name="lwaist" type="capsule" fromto="0 -.06 0 0 .06 0" size="0.05"/>
        {joint("abdomen_y", "0 0 .065")}
        <body name="pelvis" pos="0 0 -.165">
          <geom name="butt" type="capsule" fromto="-.02 -.07 0 -.02 .07 0" size="0.06"/>{leg("right", -1)}{leg("left", 1)}
        </body>
      </body>{arm("right", -1)}{arm("left", 1)}
    </body>
  </worldbody>
  <actuator>
{chr(10).join(acts)}
  </actuator>
</mujoco>
"""


# ---------------------------------------------------------------- arm + box

ARM_RANGES = ((-2.9, 2.9), (-1.7, 1.7), (-2.9, 2.9), (-3.0, -0.1), (-2.9, 2.9), (-0.1, 3.7), (-2.9, 2.9))
ARM_FINGER_RANGE = (0.0, 0.04)


def arm_xml(iterations: int = 16, tolerance: float = 1e-8, timestep: float = 0.005) -> str:
    """7-hinge arm on a table with a two-finger gripper (box palm, slide
    fingers) and a free box on the table.  The table top is the plane z = 0;
    the arm does not collide with itself; the palm box touches the object
    (box-box); the fingers are capsules (cylinder-box contacts are not in this
    build's narrowphase); the right finger mimics the left through a joint
    equality.  nq 7 + 2 + 7 = 16, nv 15, nu 9."""
    axes = ("0 0 1", "0 1 0", "0 0 1", "0 1 0", "0 0 1", "0 1 0", "0 0 1")
    links = []
    depth = 0
    for i, (ax, (lo, hi)) in enumerate(zip(axes, ARM_RANGES)):
        length = 0.16 if i % 2 == 0 else 0.14
        links.append(f"""
{'  ' * (i + 3)}<body name="link{i+1}" pos="0 0 {0.1 if i == 0 else prev_len:.3f}">
{'  ' * (i + 4)}<joint name="j{i+1}" type="hinge" axis="{ax}" range="{lo} {hi}" armature="0.05" damping="1"/>
{'  ' * (i + 4)}<geom name="link{i+1}_g" type="capsule" fromto="0 0 0 0 0 {length}" size="0.045" mass="{1.5 - 0.15*i:.2f}" contype="2" conaffinity="1"/>""")
        prev_len = length
        depth += 1
    hand = f"""
{'  ' * 10}<body name="hand" pos="0 0 {prev_len:.3f}">
{'  ' * 11}<geom name="palm" type="box" size="0.04 0.06 0.015" pos="0 0 0.015" mass="0.4" contype="2" conaffinity="1"/>
{'  ' * 11}<body name="finger_l" pos="0 0.02 0.03">
{'  ' * 12}<joint name="finger_l_j" type="slide" axis="0 1 0" range="{ARM_FINGER_RANGE[0]} {ARM_FINGER_RANGE[1]}" armature="0.01" damping="2"/>
{'  ' * 12}<geom name="finger_l_g" type="capsule" fromto="0 0 0 0 0 0.07" size="0.012" mass="0.05" contype="2" conaffinity="1"/>
{'  ' * 11}</body>
{'  ' * 11}<body name="finger_r" pos="0 -0.02 0.03">
{'  ' * 12}<joint name="finger_r_j" type="slide" axis="0 -1 0" range="{ARM_FINGER_RANGE[0]} {ARM_FINGER_RANGE[1]}" armature="0.01" damping="2"/>
{'  ' * 12}<geom name="finger_r_g" type="capsule" fromto="0 0 0 0 0 0.07" size="0.012" mass="0.05" contype="2" conaffinity="1"/>
{'  ' * 11}</body>
{'  ' * 10}</body>"""
    closes = "".join(f"\n{'  ' * (i + 3)}</body>" for i in reversed(range(7)))
    acts = [f'    <position name="j{i+1}_act" joint="j{i+1}" kp="80" kv="4" ctrlrange="{lo} {hi}"/>' for i, (lo, hi) in enumerate(ARM_RANGES)]
    acts += [f'    <position name="{f}_act" joint="{f}_j" kp="40" kv="1" ctrlrange="{ARM_FINGER_RANGE[0]} {ARM_FINGER_RANGE[1]}"/>'
             for f in ("finger_l", "finger_r")]
    return f"""<mujoco model="arm7_gripper_box">
  <compiler angle="radian"/>
  <option timestep="{timestep}" iterations="{iterations}" tolerance="{tolerance}" cone="pyramidal" integrator="Euler"/>
  <default><geom condim="3" friction="1 0.005 0.0001"/></default>
  <worldbody>
    <geom name="table" type="plane" size="0 0 1"/>
    <body name="base" pos="0 0 0">
      <geom name="base_g" type="box" size="0.08 0.08 0.05" pos="0 0 0.05" mass="5" contype="2" conaffinity="0"/>{''.join(links)}{hand}{closes}
    </body>
    <body name="object" pos="0.45 0 0.03">
      <freejoint name="object_root"/>
      <geom name="object_g" type="box" size="0.03 0.03 0.03" mass="0.2"/>
    </body>
  </worldbody>
  <equality>
    <joint name="finger_mimic" joint1="finger_r_j" joint2="finger_l_j" polycoef="0 1 0 0 0"/>
  </equality>
  <actuator>
{chr(10).join(acts)}
  </actuator>
</mujoco>
"""


def joint_ranges(model) -> np.ndarray:
    """Ranges [nu, 2] of the joints (or fixed tendons) the model's actuators
    drive, as position targets; an unlimited tendon gets [-0.2, 0.2]."""
    d = model.dump()
    trn = d["actuator_trnid"]
    kind = d.get("actuator_trntype", np.zeros_like(trn))
    rng = d["jnt_range"].reshape(-1, 2)
    out = np.zeros((len(trn), 2))
    for a, (k, i) in enumerate(zip(kind, trn)):
        if k == 3:
            out[a] = d["tendon_range"].reshape(-1, 2)[i] if d["tendon_limited"][i] else (-0.2, 0.2)
        else:
            out[a] = rng[i]
    return out


def random_state(model, num_envs: int, seed: int, height=None, noise: float = 0.1):
    """qpos0 plus N(0, noise) on hinge/slide joints (clipped to their ranges),
    an optional root height range for a free root, zero velocity."""
    d = model.dump()
    g = np.random.Generator(np.random.Philox(key=seed))
    q0 = d["qpos0"].astype(np.float64)
    qpos = np.tile(q0, (num_envs, 1))
    jt, qa, lim = d["jnt_type"], d["jnt_qposadr"], d["jnt_limited"]
    rng = d["jnt_range"].reshape(-1, 2)
    for j in range(len(jt)):
        if jt[j] in (2, 3):
            a = qa[j]
            lo, hi = rng[j] if lim[j] else (-np.inf, np.inf)
            centre = 0.0 if lo <= 0.0 <= hi else 0.5 * (lo + hi)
            qpos[:, a] = np.clip(centre + g.normal(0.0, noise, size=num_envs), lo, hi)
    if height is not None and len(jt) and jt[0] == 0:
        qpos[:, 2] = g.uniform(height[0], height[1], size=num_envs)
    return qpos, np.zeros((num_envs, model.nv))


def random_controls(model, num_envs: int, step: int, seed: int):
    """Position targets U[joint range] for control step `step`."""
    r = joint_ranges(model)
    g = np.random.Generator(np.random.Philox(key=seed, counter=step))
    return r[:, 0] + (r[:, 1] - r[:, 0]) * g.random((num_envs, len(r)))


# ---------------------------------------------------------------- hinge chains

CHAIN_LINK = 0.1


def chain_xml(n: int, cfg: str, iterations: int = 50) -> str:
    """Pendulum chain of n hinge links (alternating y / x axes, capsules of
    0.1 m, joint damping 0.02) for robustness sweeps over the dof count, in
    the spirit of the reference's tests/test_robustness.cpp.  cfg:
    "free" (no collision pairs), "limit" (joint limits +-0.35 rad), "floss"
    (frictionloss 0.05), "contact" (floor touched when the first joint swings
    1.2 rad), "all" (limits, frictionloss and contact), "equality" (every
    odd joint coupled to 0.5 x the previous joint by a joint equality)."""
    H = n * CHAIN_LINK + 0.05
    touch = H - n * CHAIN_LINK * math.cos(1.2) - 0.004
    floor_z = touch if cfg in ("contact", "all") else -50.0
    floor_col = ' contype="0" conaffinity="0"' if cfg == "free" else ""
    jattr = ""
    if cfg in ("limit", "all"):
        jattr += ' limited="true" range="-0.35 0.35"'
    if cfg in ("floss", "all"):
        jattr += ' frictionloss="0.05"'
    gcol = ' contype="0" conaffinity="0"' if cfg == "free" else ' contype="1" conaffinity="1"'
    body = []
    for i in range(n):
        axis = "1 0 0" if i % 2 else "0 1 0"
        z = H if i == 0 else -CHAIN_LINK
        body.append(f'<body pos="0 0 {z:.4f}"><joint name="j{i}" type="hinge" axis="{axis}" damping="0.02"{jattr}/>'
                    f'<geom type="capsule" fromto="0 0 0 0 0 {-CHAIN_LINK}" size="0.02" density="500"{gcol}/>')
    eq = ""
    if cfg == "equality":
        eq = "<equality>" + "".join(f'<joint joint1="j{i}" joint2="j{i - 1}" polycoef="0 0.5 0 0 0"/>' for i in range(1, n, 2)) + "</equality>"
    return (f'<mujoco model="chain{n}_{cfg}"><compiler angle="radian"/>'
            f'<option timestep="0.002" iterations="{iterations}" tolerance="1e-8" cone="pyramidal" integrator="Euler"/>'
            f'<worldbody><geom type="plane" size="5 5 0.1" pos="0 0 {floor_z:.4f}"{floor_col}/>'
            + "".join(body) + "</body>" * n + "</worldbody>" + eq + "</mujoco>")


def tendon_chain_xml(n: int = 8, iterations: int = 50) -> str:
    """Hinge chain (as chain_xml, n >= 8, no contact) coupled by fixed
    tendons: t0 = j0 + 0.5 j1 (limited +-0.3, frictionloss, spring with a
    dead band, damper), t1 = j2 - j3 + 0.5 j4 (auto-limited +-0.4, margin
    0.02), t2 = j1 + j5 (frictionloss, spring to its rest length), t3, t4
    held by a tendon equality t3 - t3_0 = 0.8 (t4 - t4_0); a motor on t0 and
    a position actuator (kp 5) on t1."""
    assert n >= 8
    H = n * CHAIN_LINK + 0.05
    body = []
    for i in range(n):
        axis = "1 0 0" if i % 2 else "0 1 0"
        z = H if i == 0 else -CHAIN_LINK
        body.append(f'<body pos="0 0 {z:.4f}"><joint name="j{i}" type="hinge" axis="{axis}" damping="0.02"/>'
                    f'<geom type="capsule" fromto="0 0 0 0 0 {-CHAIN_LINK}" size="0.02" density="500" contype="0" conaffinity="0"/>')
    ten = ('<tendon>'
           '<fixed name="t0" limited="true" range="-0.3 0.3" frictionloss="0.03" stiffness="2" springlength="-0.05 0.05" damping="0.05">'
           '<joint joint="j0" coef="1"/><joint joint="j1" coef="0.5"/></fixed>'
           '<fixed name="t1" range="-0.4 0.4" margin="0.02"><joint joint="j2" coef="1"/><joint joint="j3" coef="-1"/><joint joint="j4" coef="0.5"/></fixed>'
           '<fixed name="t2" frictionloss="0.02" stiffness="1"><joint joint="j1" coef="1"/><joint joint="j5" coef="1"/></fixed>'
           '<fixed name="t3"><joint joint="j6" coef="1"/><joint joint="j7" coef="0.7"/></fixed>'
           '<fixed name="t4"><joint joint="j4" coef="1"/><joint joint="j5" coef="-0.3"/></fixed>'
           '</tendon>')
    eq = '<equality><tendon tendon1="t3" tendon2="t4" polycoef="0 0.8 0 0 0"/></equality>'
    act = ('<actuator><motor tendon="t0" gear="1" ctrllimited="true" ctrlrange="-1 1"/>'
           '<position tendon="t1" kp="5"/></actuator>')
    return (f'<mujoco model="tendon_chain{n}"><compiler angle="radian"/>'
            f'<option timestep="0.002" iterations="{iterations}" tolerance="1e-8" cone="pyramidal" integrator="Euler"/>'
            '<worldbody>' + "".join(body) + "</body>" * n + "</worldbody>" + ten + eq + act + "</mujoco>")


def sensor_xml(floor: bool = False) -> str:
    """Floating torso with an IMU site (tilted), a two-hinge arm with a tip
    site, a slider, a ball-jointed pendulum and a fixed tendon over the arm
    hinges; motors, a position actuator and a tendon motor; one sensor of
    every type in the batched set, plus a touch sensor and a relative frame
    sensor (outside the set, read as zeros).  floor: a collidable plane
    under the torso (otherwise the robot floats in free fall)."""
    plane = '<geom name="floor" type="plane" size="5 5 0.1" pos="0 0 -0.2"/>' if floor else ""
    return (
        '<mujoco model="sensor_rig"><compiler angle="radian"/>'
        '<option timestep="0.004" iterations="30" tolerance="1e-8" integrator="Euler" magnetic="0.1 -0.4 0.3"/>'
        '<worldbody>' + plane +
        '<body name="torso" pos="0 0 0.4"><freejoint/>'
        '<geom name="torso_g" type="box" size="0.12 0.08 0.04" mass="1.5"/>'
        '<site name="imu" pos="0.02 -0.01 0.03" euler="0.2 0.4 -0.3"/>'
        '<body name="arm" pos="0.12 0 0"><joint name="shoulder" type="hinge" axis="0 1 0" damping="0.05"/>'
        '<geom name="arm_g" type="capsule" fromto="0 0 0 0.18 0 0" size="0.02" mass="0.25"/>'
        '<site name="tip" pos="0.18 0 0" quat="0.8 0.6 0 0"/>'
        '<body name="fore" pos="0.18 0 0"><joint name="elbow" type="hinge" axis="0 1 0" damping="0.05"/>'
        '<geom name="fore_g" type="capsule" fromto="0 0 0 0.12 0 0" size="0.015" mass="0.15"/></body></body>'
        '<body name="slider" pos="-0.12 0 0"><joint name="slide" type="slide" axis="0 0 1" range="-0.08 0.08" damping="0.4"/>'
        '<geom name="slider_g" type="sphere" size="0.025" mass="0.2" pos="0.01 0 0"/>'
        '<site name="slider_site" pos="0 0.01 -0.025"/></body>'
        '<body name="pend" pos="0 0.1 0"><joint name="ballj" type="ball" damping="0.01"/>'
        '<geom name="pend_g" type="box" size="0.015 0.015 0.04" pos="0 0 -0.04" mass="0.2"/></body>'
        '</body></worldbody>'
        '<tendon><fixed name="tsum"><joint joint="shoulder" coef="1"/><joint joint="elbow" coef="0.5"/></fixed></tendon>'
        '<actuator><motor name="m_sh" joint="shoulder" gear="2"/><motor name="m_el" joint="elbow"/>'
        '<position name="p_sl" joint="slide" kp="15" gear="1.5"/><motor name="m_t" tendon="tsum" gear="0.5"/></actuator>'
        '<sensor>'
        '<gyro name="imu_gyro" site="imu"/><accelerometer name="imu_acc" site="imu"/><velocimeter name="imu_vel" site="imu"/>'
        '<magnetometer name="imu_mag" site="imu"/><accelerometer name="tip_acc" site="tip"/><gyro name="tip_gyro" site="tip"/>'
        '<framepos name="imu_pos" objtype="site" objname="imu"/><framequat name="imu_quat" objtype="site" objname="imu"/>'
        '<framexaxis name="tip_x" objtype="site" objname="tip"/><frameyaxis name="tip_y" objtype="site" objname="tip"/>'
        '<framezaxis name="tip_z" objtype="site" objname="tip"/><framelinvel name="tip_v" objtype="site" objname="tip"/>'
        '<frameangvel name="tip_w" objtype="site" objname="tip"/><framepos name="arm_ipos" objtype="body" objname="arm"/>'
        '<framequat name="arm_iquat" objtype="body" objname="arm"/><framelinvel name="fore_v" objtype="body" objname="fore"/>'
        '<framepos name="fore_xpos" objtype="xbody" objname="fore"/><framequat name="fore_gq" objtype="geom" objname="fore_g"/>'
        '<framepos name="slider_gp" objtype="geom" objname="slider_g"/>'
        '<jointpos name="q_sh" joint="shoulder"/><jointvel name="v_sh" joint="shoulder"/><jointpos name="q_sl" joint="slide"/>'
        '<jointvel name="v_sl" joint="slide"/><jointactuatorfrc name="f_sh" joint="shoulder"/><jointactuatorfrc name="f_sl" joint="slide"/>'
        '<ballquat name="ball_q" joint="ballj"/><ballangvel name="ball_w" joint="ballj"/>'
        '<actuatorpos name="ap_sh" actuator="m_sh"/><actuatorvel name="av_sh" actuator="m_sh"/>'
        '<actuatorpos name="ap_t" actuator="m_t"/><actuatorvel name="av_t" actuator="m_t"/>'
        '<tendonpos name="t_pos" tendon="tsum"/><tendonvel name="t_vel" tendon="tsum"/>'
        '<subtreecom name="com" body="torso"/><subtreecom name="arm_com" body="arm"/>'
        '<touch name="touch_tip" site="tip"/><framepos name="rel_pos" objtype="site" objname="tip" reftype="body" refname="torso"/>'
        '</sensor></mujoco>')


def sensor_state(model, num_envs: int, seed: int, qnoise: float = 0.3, vnoise: float = 1.0):
    """qpos0 with N(0, qnoise) on the hinges, slide and ball (renormalised),
    the free root rotated by up to 0.5 rad; N(0, vnoise) velocities."""
    d = model.dump()
    g = np.random.Generator(np.random.Philox(key=seed))
    q = np.tile(d["qpos0"].astype(np.float64), (num_envs, 1))
    jt, qa = d["jnt_type"], d["jnt_qposadr"]
    for j in range(len(jt)):
        a = qa[j]
        if jt[j] in (2, 3):
            q[:, a] += g.normal(0, qnoise, num_envs)
            if jt[j] == 2:
                q[:, a] = np.clip(q[:, a], -0.07, 0.07)
        else:
            o = a + 3 if jt[j] == 0 else a
            ax = g.normal(size=(num_envs, 3))
            ax /= np.linalg.norm(ax, axis=1, keepdims=True)
            ang = g.uniform(0, 0.5, num_envs)
            q[:, o] = np.cos(ang / 2)
            q[:, o + 1: o + 4] = ax * np.sin(ang / 2)[:, None]
    v = g.normal(0, vnoise, size=(num_envs, model.nv))
    return q, v


def spatial_tendon_xml(iterations: int = 50) -> str:
    """Two-link arm (shoulder and elbow hinges about y) on a fixed base with
    spatial tendons: 'flexor' runs from the base over a wrapping sphere at the
    shoulder, a site on the upper arm, around a wrapping cylinder at the elbow
    (with a side site) to the forearm (limited, spring, damper, frictionloss);
    'rope' hangs a slider from a world site through a pulley (divisor 2)
    shared with the forearm tip; 'strap' is a straight site-to-site tendon.
    A motor pulls on the flexor, a position actuator on the slider."""
    return (
        '<mujoco model="spatial_tendons"><compiler angle="radian"/>'
        f'<option timestep="0.002" iterations="{iterations}" tolerance="1e-8" integrator="Euler"/>'
        '<worldbody>'
        '<site name="top" pos="0.35 0 0.9"/>'
        '<body name="base" pos="0 0 0.6">'
        '<geom type="box" size="0.05 0.05 0.05" contype="0" conaffinity="0" mass="2"/>'
        '<site name="origin" pos="-0.02 0 0.18"/>'
        '<geom name="shoulder_wrap" type="sphere" size="0.06" pos="0 0 0.08" contype="0" conaffinity="0" mass="0.01"/>'
        '<body name="upper" pos="0 0 0.08"><joint name="shoulder" type="hinge" axis="0 1 0" damping="0.1"/>'
        '<geom type="capsule" fromto="0 0 0 0.3 0 0" size="0.025" contype="0" conaffinity="0" mass="0.8"/>'
        '<site name="mid" pos="0.15 0 0.05"/>'
        '<geom name="elbow_wrap" type="cylinder" size="0.04 0.03" pos="0.3 0 0" quat="0.7071068 0.7071068 0 0" contype="0" conaffinity="0" mass="0.01"/>'
        '<site name="elbow_side" pos="0.3 0 0.1"/>'
        '<body name="fore" pos="0.3 0 0"><joint name="elbow" type="hinge" axis="0 1 0" damping="0.1"/>'
        '<geom type="capsule" fromto="0 0 0 0.25 0 0" size="0.02" contype="0" conaffinity="0" mass="0.5"/>'
        '<site name="insert" pos="0.12 0 0.02"/><site name="tip" pos="0.25 0 0"/></body></body></body>'
        '<body name="slider" pos="0.6 0 0.5"><joint name="slide" type="slide" axis="0 0 1" damping="0.5"/>'
        '<geom type="sphere" size="0.03" contype="0" conaffinity="0" mass="0.3"/><site name="hook" pos="0 0 0.03"/></body>'
        '</worldbody>'
        '<tendon>'
        '<spatial name="flexor" limited="true" range="0.435 0.46" stiffness="30" damping="0.5" frictionloss="0.05">'
        '<site site="origin"/><geom geom="shoulder_wrap"/><site site="mid"/><geom geom="elbow_wrap" sidesite="elbow_side"/><site site="insert"/>'
        '</spatial>'
        '<spatial name="rope" stiffness="100" springlength="0.55">'
        '<site site="tip"/><site site="top"/><pulley divisor="2"/><site site="top"/><site site="hook"/></spatial>'
        '<spatial name="strap" frictionloss="0.02" range="0.5 0.56"><site site="origin"/><site site="tip"/></spatial>'
        '</tendon>'
        '<actuator><motor name="pull" tendon="flexor" gear="5" ctrllimited="true" ctrlrange="-1 1"/>'
        '<position name="lift" joint="slide" kp="20"/></actuator>'
        '</mujoco>')


def chain_state(n: int, cfg: str, num_envs: int, seed: int):
    """Random joint angles N(0, 0.5) (beyond the limits for some envs), the
    first joint swung by 1.2 rad for contact configurations, random joint
    velocities N(0, 0.5)."""
    g = np.random.Generator(np.random.Philox(key=seed))
    q = g.normal(0.0, 0.5, size=(num_envs, n))
    if cfg in ("contact", "all"):
        q[:, 0] += 1.2
    v = g.normal(0.0, 0.5, size=(num_envs, n))
    return q, v


# ---------------------------------------------------------------- box pile

def box_pile_xml(nbox: int = 4, seed: int = 0, iterations: int = 30) -> str:
    """nbox free boxes (half sizes U[0.04, 0.12], masses U[0.2, 1.0] kg)
    stacked loosely above a plane, for box-box / box-plane contacts."""
    g = np.random.Generator(np.random.Philox(key=seed))
    bodies = []
    z = 0.0
    for i in range(nbox):
        h = g.uniform(0.04, 0.12, size=3)
        z += h[2] + 0.01
        x, y = g.uniform(-0.05, 0.05, size=2)
        bodies.append(f'<body name="box{i}" pos="{x:.4f} {y:.4f} {z:.4f}"><freejoint/>'
                      f'<geom type="box" size="{h[0]:.4f} {h[1]:.4f} {h[2]:.4f}" mass="{g.uniform(0.2, 1.0):.3f}"/></body>')
        z += h[2]
    return (f'<mujoco model="box_pile{nbox}"><compiler angle="radian"/>'
            f'<option timestep="0.005" iterations="{iterations}" tolerance="1e-8" cone="pyramidal" integrator="Euler"/>'
            '<default><geom condim="3" friction="0.8 0.005 0.0001"/></default>'
            '<worldbody><geom name="floor" type="plane" size="0 0 1"/>' + "".join(bodies) + '</worldbody></mujoco>')


def noisy_sphere_vertices(npts: int, radius: float, noise: float, g) -> np.ndarray:
    """npts points on a sphere of the given radius, each radius x U[1 -
    noise, 1 + noise] (a rock-like convex hull)."""
    d = g.normal(size=(npts, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return d * (radius * g.uniform(1 - noise, 1 + noise, size=(npts, 1)))


CONVEX_SHAPES = ("ellipsoid", "cylinder", "mesh", "capsule", "sphere", "box")


def convex_pile_xml(nbody: int = 6, seed: int = 0, iterations: int = 30, condim: int = 3, cone: str = "pyramidal") -> str:
    """nbody free bodies cycling through ellipsoid, cylinder, 32-point noisy
    sphere hull (r = 0.05 +- 20 %), capsule, sphere and box (sizes about
    0.04-0.06 m), stacked loosely in a 0.1 m column above a plane, for the
    GJK / EPA convex pairs (the bin workload's shapes at a size the dense
    solver holds: nv = 6 nbody <= 64)."""
    g = np.random.Generator(np.random.Philox(key=seed))
    assets, bodies = [], []
    z = 0.0
    for i in range(nbody):
        kind = CONVEX_SHAPES[i % len(CONVEX_SHAPES)]
        if kind == "ellipsoid":
            a = g.uniform(0.03, 0.06, 3)
            geom, h = f'type="ellipsoid" size="{a[0]:.4f} {a[1]:.4f} {a[2]:.4f}"', a.max()
        elif kind == "cylinder":
            r, hh = g.uniform(0.03, 0.05), g.uniform(0.03, 0.05)
            geom, h = f'type="cylinder" size="{r:.4f} {hh:.4f}"', max(r, hh)
        elif kind == "mesh":
            v = noisy_sphere_vertices(32, 0.05, 0.2, g)
            assets.append(f'<mesh name="rock{i}" vertex="' + " ".join(f"{x:.5f}" for x in v.reshape(-1)) + '"/>')
            geom, h = f'type="mesh" mesh="rock{i}"', 0.06
        elif kind == "capsule":
            r, hh = g.uniform(0.02, 0.035), g.uniform(0.03, 0.05)
            geom, h = f'type="capsule" size="{r:.4f} {hh:.4f}"', r + hh
        elif kind == "sphere":
            r = g.uniform(0.03, 0.05)
            geom, h = f'type="sphere" size="{r:.4f}"', r
        else:
            a = g.uniform(0.025, 0.045, 3)
            geom, h = f'type="box" size="{a[0]:.4f} {a[1]:.4f} {a[2]:.4f}"', np.linalg.norm(a)
        z += h + 0.002
        x, y = g.uniform(-0.03, 0.03, 2)
        bodies.append(f'<body name="b{i}" pos="{x:.4f} {y:.4f} {z:.4f}"><freejoint/><geom {geom} mass="{g.uniform(0.1, 0.4):.3f}"/></body>')
        z += h
    return (f'<mujoco model="convex_pile{nbody}"><compiler angle="radian"/>'
            f'<option timestep="0.004" iterations="{iterations}" tolerance="1e-8" cone="{cone}" integrator="Euler"/>'
            f'<default><geom condim="{condim}" friction="0.7 0.01 0.001"/></default>'
            + (f'<asset>{"".join(assets)}</asset>' if assets else "")
            + '<worldbody><geom name="floor" type="plane" size="0 0 1"/>' + "".join(bodies) + '</worldbody></mujoco>')


def pushed_box_xml(cone: str = "elliptic", condim: int = 3, mu: float = 0.5, impratio: float = 1.0) -> str:
    """A 1 kg cube (half size 0.1 m) on a plane, on three slide joints (x,
    y, z) and a ball joint, with a motor on the x slide: the friction-cone
    known-answer model (sticks for pushes below mu m g, slides above).
    Tangential friction mu, torsional 0.02, rolling 0.002; dt 0.002."""
    fr = f'friction="{mu} 0.02 0.002" condim="{condim}"'
    return (f'<mujoco model="pushed_box"><option timestep="0.002" iterations="100" tolerance="1e-10" cone="{cone}" impratio="{impratio}"/>'
            f'<worldbody><geom name="floor" type="plane" size="0 0 1" {fr}/>'
            f'<body name="box" pos="0 0 0.1"><joint name="sx" type="slide" axis="1 0 0"/><joint name="sy" type="slide" axis="0 1 0"/>'
            f'<joint name="sz" type="slide" axis="0 0 1"/><joint name="rot" type="ball"/>'
            f'<geom type="box" size="0.1 0.1 0.1" mass="1" {fr}/></body></worldbody>'
            f'<actuator><motor name="push" joint="sx"/></actuator></mujoco>')


BIN_SHAPES = ("box", "capsule", "ellipsoid", "mesh")


def bin_xml(nbody: int = 64, size: float = 1.0, seed: int = 0, condim: int = 3, iterations: int = 30, cone: str = "pyramidal") -> str:
    """A square bin (floor plus four inward-facing wall planes, side `size`)
    holding nbody free bodies cycling through boxes, capsules, ellipsoids and
    convex hulls of 32 points on a 0.05 m sphere with +-20 % radial noise,
    placed on a jittered grid in layers above the floor with random
    orientations (the collision-heavy bin workload; nv = 6 nbody)."""
    g = np.random.Generator(np.random.Philox(key=seed))
    half = 0.5 * size
    walls = ['<geom name="floor" type="plane" size="0 0 1"/>']
    for k, (x, y, zx) in enumerate([(half, 0, "-1 0 0"), (-half, 0, "1 0 0"), (0, half, "0 -1 0"), (0, -half, "0 1 0")]):
        walls.append(f'<geom name="wall{k}" type="plane" pos="{x:.4f} {y:.4f} 0" zaxis="{zx}" size="{half:.4f} {half:.4f} 0.1"/>')
    per_side = max(1, int(np.ceil(np.sqrt(min(nbody, 16)))))
    pitch = (size - 0.16) / max(per_side - 1, 1) if per_side > 1 else 0.0
    assets, bodies = [], []
    for i in range(nbody):
        kind = BIN_SHAPES[i % len(BIN_SHAPES)]
        if kind == "box":
            a = g.uniform(0.025, 0.045, 3)
            geom = f'type="box" size="{a[0]:.4f} {a[1]:.4f} {a[2]:.4f}"'
        elif kind == "capsule":
            geom = f'type="capsule" size="{g.uniform(0.02, 0.03):.4f} {g.uniform(0.03, 0.045):.4f}"'
        elif kind == "ellipsoid":
            a = g.uniform(0.03, 0.055, 3)
            geom = f'type="ellipsoid" size="{a[0]:.4f} {a[1]:.4f} {a[2]:.4f}"'
        else:
            v = noisy_sphere_vertices(32, 0.05, 0.2, g)
            assets.append(f'<mesh name="hull{i}" vertex="' + " ".join(f"{x:.5f}" for x in v.reshape(-1)) + '"/>')
            geom = f'type="mesh" mesh="hull{i}"'
        layer, cell = divmod(i, per_side * per_side)
        cx, cy = divmod(cell, per_side)
        x = -half + 0.08 + cx * pitch + g.uniform(-0.02, 0.02)
        y = -half + 0.08 + cy * pitch + g.uniform(-0.02, 0.02)
        z = 0.08 + 0.14 * layer + g.uniform(0.0, 0.02)
        q = g.normal(size=4)
        q /= np.linalg.norm(q)
        bodies.append(f'<body name="b{i}" pos="{x:.4f} {y:.4f} {z:.4f}" quat="{q[0]:.5f} {q[1]:.5f} {q[2]:.5f} {q[3]:.5f}"><freejoint/>'
                      f'<geom {geom} mass="{g.uniform(0.1, 0.5):.3f}"/></body>')
    return (f'<mujoco model="bin{nbody}"><compiler angle="radian"/>'
            f'<option timestep="0.004" iterations="{iterations}" tolerance="1e-8" cone="{cone}" integrator="Euler"/>'
            f'<default><geom condim="{condim}" friction="0.8 0.01 0.001"/></default>'
            + (f'<asset>{"".join(assets)}</asset>' if assets else "")
            + '<worldbody>' + "".join(walls) + "".join(bodies) + '</worldbody></mujoco>')


def box_pile_state(model, num_envs: int, seed: int):
    """qpos0 with each box's position jittered by U[-0.03, 0.03] m and its
    orientation rotated by up to 0.4 rad about a random axis."""
    d = model.dump()
    g = np.random.Generator(np.random.Philox(key=seed))
    q0 = d["qpos0"].astype(np.float64)
    nb = model.nq // 7
    qpos = np.tile(q0, (num_envs, 1))
    for b in range(nb):
        a = 7 * b
        qpos[:, a:a + 3] += g.uniform(-0.03, 0.03, size=(num_envs, 3))
        ax = g.normal(size=(num_envs, 3))
        ax /= np.linalg.norm(ax, axis=1, keepdims=True)
        ang = g.uniform(0.0, 0.4, size=num_envs)
        qpos[:, a + 3] = np.cos(ang / 2)
        qpos[:, a + 4:a + 7] = ax * np.sin(ang / 2)[:, None]
    return qpos, np.zeros((num_envs, model.nv))
