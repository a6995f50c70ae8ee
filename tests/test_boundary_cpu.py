"""Host-side parts of the drop-in boundary that need no GPU: the torch.ops.vpt registrations
(Module.cpp:186-280) and the environment-map rotation matrices of the module's setters
(RotationWidget::getMat3, src/Utils/RotationWidget.cpp:62-77: glm::eulerAngleYXZ, glm::yawPitchRoll,
glm::angleAxis, glm::toMat3), checked against scipy's rotations."""
import math

import numpy as np
import pytest
import torch
from scipy.spatial.transform import Rotation

from cloudrendering_b200 import torch_ops, vpt


def test_every_operator_is_registered_with_its_schema():
    for name in torch_ops.OPS:
        op = getattr(torch.ops.vpt, name)
        assert str(op.default._schema) == "vpt::" + torch_ops.schema(name, getattr(vpt, name))
    assert str(torch.ops.vpt.render_frame.default._schema) == \
        "vpt::render_frame(Tensor input_tensor, int frame_count) -> Tensor"
    assert str(torch.ops.vpt.set_global_world_bounding_box.default._schema) == \
        "vpt::set_global_world_bounding_box(float[] global_bb_vec) -> ()"


def test_operator_reaches_the_module_function(monkeypatch):
    seen = []
    monkeypatch.setattr(vpt, "_c", lambda name, *args: seen.append(name))
    torch.ops.vpt.set_seed_offset(7)
    torch.ops.vpt.disable_env_map_rot()
    assert seen == ["vpt_set_seed_offset", "vpt_set_env_map_rotation"]


@pytest.fixture
def captured(monkeypatch):
    box = {}

    def grab(name, *args):
        if name == "vpt_set_env_map_rotation":
            box["m"] = np.array(list(args[0]), np.float64).reshape(3, 3).T  # column-major -> row-major
    monkeypatch.setattr(vpt, "_c", grab)
    return box


def test_euler_angles_are_yxz(captured):
    a, b, c = 0.7, -0.4, 0.25
    vpt.set_env_map_rot_euler_angles([a, b, c])
    want = Rotation.from_euler("YXZ", [a, b, c]).as_matrix()  # intrinsic: Ry(a) Rx(b) Rz(c)
    assert np.allclose(captured["m"], want, atol=1e-6)
    vpt.set_env_map_rot_yaw_pitch_roll([a, b, c])  # glm::yawPitchRoll is the same matrix
    assert np.allclose(captured["m"], want, atol=1e-6)


def test_angle_axis_and_quaternion(captured):
    axis, angle = np.array([0.3, -1.0, 0.5]), 1.1
    vpt.set_env_map_rot_angle_axis(list(axis), angle)
    want = Rotation.from_rotvec(axis / np.linalg.norm(axis) * angle).as_matrix()
    assert np.allclose(captured["m"], want, atol=1e-6)
    q = Rotation.from_rotvec([0.2, 0.4, -0.3]).as_quat()  # (x, y, z, w), the order of parseQuaternion
    vpt.set_env_map_rot_quaternion(list(q))
    assert np.allclose(captured["m"], Rotation.from_quat(q).as_matrix(), atol=1e-6)
    with pytest.raises(RuntimeError):
        vpt.set_env_map_rot_quaternion([0.0, 0.0, 1.0])


def test_rotation_matrices_are_orthonormal(captured):
    vpt.set_env_map_rot_angle_axis([0.0, 0.0, 2.0], math.pi / 3)
    m = captured["m"]
    assert np.allclose(m @ m.T, np.eye(3), atol=1e-6)
    assert np.allclose(m, Rotation.from_euler("z", math.pi / 3).as_matrix(), atol=1e-6)


def test_transfer_function_empty_and_albedo_strength(monkeypatch):
    """set_transfer_function_empty uploads the reference's empty function (opacity and colour 0 at both
    ends, Module.cpp:1262-1276); set_tf_scattering_albedo_strength forwards its weight."""
    seen = []

    def grab(name, *args):
        if name == "vpt_set_transfer_function":
            ptr, n = args
            import ctypes
            seen.append((name, np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), (n * 4,)).copy()))
        else:
            seen.append((name, args))
    monkeypatch.setattr(vpt, "_c", grab)
    vpt.set_transfer_function_empty()
    torch.ops.vpt.set_tf_scattering_albedo_strength(0.75)
    assert seen[0][0] == "vpt_set_transfer_function" and np.array_equal(seen[0][1], np.zeros(8, np.float32))
    assert seen[1] == ("vpt_set_tf_scattering_albedo_strength", (0.75,))
