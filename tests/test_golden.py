"""The FP64 oracle against its committed regression fixtures
(tests/golden/quadruped16.npz, written by tests/golden/make_golden.py).

The fixtures are the oracle's own outputs on the seeded 16-env quadruped
workload with the committed model dump, not outputs of the reference: they
catch unintended changes to the oracle, the dump or the seeded inputs.
"""
import os

import numpy as np
import pytest

import oracle
from mjb200 import models

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(HERE, "golden", "quadruped16.npz")))


@pytest.fixture(scope="module")
def om():
    return oracle.OracleModel(oracle.load_dump("quadruped12.dump"))


def test_inputs_are_the_seeded_workload(gold):
    B = gold["q0"].shape[0]
    q0, v0 = models.quadruped_initial_state(B)
    np.testing.assert_array_equal(gold["q0"], q0)
    np.testing.assert_array_equal(gold["v0"], v0)
    for k in range(2):
        np.testing.assert_array_equal(gold["ctrl"][k], models.quadruped_controls(B, k))
    np.testing.assert_array_equal(gold["cs"], models.quadruped_controls(B, 25))


def test_two_control_steps_match(gold, om):
    B = gold["q0"].shape[0]
    for e in range(B):
        env = oracle.OracleEnv(om, 64, 128)
        env.a["qpos"][:] = gold["q0"][e]
        env.a["qvel"][:] = gold["v0"][e]
        for k in range(2):
            env.a["ctrl"][:12] = gold["ctrl"][k][e]
            for _ in range(4):
                env.step()
            np.testing.assert_allclose(env.a["qpos"], gold[f"q{k + 1}"][e], rtol=0, atol=1e-10, err_msg=f"env {e} step {k}")
            np.testing.assert_allclose(env.a["qvel"], gold[f"v{k + 1}"][e], rtol=0, atol=1e-8, err_msg=f"env {e} step {k}")


def test_one_substep_at_the_settled_state_matches(gold, om):
    B = gold["qs"].shape[0]
    assert gold["ncon"].max() > 0
    for e in range(B):
        env = oracle.OracleEnv(om, 64, 128)
        env.a["qpos"][:] = gold["qs"][e]
        env.a["qvel"][:] = gold["vs"][e]
        env.a["ctrl"][:12] = gold["cs"][e]
        env.step()
        ncon, nefc = env.d.ncon, env.d.nefc
        assert (ncon, nefc, env.d.niter) == (gold["ncon"][e], gold["nefc"][e], gold["niter"][e]), e
        np.testing.assert_array_equal(env.contacts()[:, 13].astype(np.int32), gold["pairs"][e][:ncon])
        efc = env.efc()
        np.testing.assert_array_equal(efc["type"], gold["efc_type"][e][:nefc])
        scale = max(1.0, np.abs(gold["efc_force"][e]).max())
        np.testing.assert_allclose(efc["force"], gold["efc_force"][e][:nefc], rtol=0, atol=1e-9 * scale)
        np.testing.assert_allclose(env.a["qacc"], gold["qacc"][e], rtol=1e-9, atol=1e-9)
