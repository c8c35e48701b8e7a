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
