"""Service-layer contracts on CPU: lifecycle, scene registries, owned outputs,
render cadence and the reference's error texts.

The services are driven with ``allow_cpu_for_tests=True`` and a recording
backend, the way the reference's own service tests drive theirs
(tests/test_renderer_service.py, tests/test_lidar_service.py of the
reference): nothing here renders.
"""

from __future__ import annotations

import pytest
import torch

from vgr_b200 import RendererService
from vgr_b200.lidar_scene import GaussianLidarScene, LidarSceneRegistry
from vgr_b200.lidar_service import GaussianLidarService
from vgr_b200.scene import GaussianScene, SceneRegistry

CPU = torch.device("cpu")


class RecordingBackend:
    """Writes the request's camera count into every float output."""

    def __init__(self) -> None:
        self.calls: list[str] = []
        self.scenes: list[tuple[int, int]] = []

    def initialize(self, stage, device) -> None:
        self.calls.append("initialize")

    def allocate_workspace(self, **kwargs):
        self.calls.append("allocate_workspace")
        return {"marker": torch.zeros(1)}

    def register_scene(self, scene_id, scene, offset) -> None:
        self.scenes.append((scene_id, offset))

    def update_scene_transforms(self, scene_ids, transforms) -> None:
        self.calls.append("update")

    def render(self, request) -> None:
        self.calls.append("render")
        for name, tensor in request.outputs.items():
            if tensor.is_floating_point():
                tensor.fill_(float(request.camera_transforms.shape[0]))

    def synchronize(self) -> None:
        self.calls.append("synchronize")

    def shutdown(self) -> None:
        self.calls.append("shutdown")


def scene_kwargs(count: int = 2) -> dict[str, torch.Tensor]:
    return {
        "means": torch.zeros((count, 3)),
        "scales": torch.ones((count, 3)),
        "rotations": torch.tensor([[1.0, 0.0, 0.0, 0.0]] * count),
        "opacities": torch.ones((count,)),
        "features": torch.ones((count, 3)),
        "semantic_ids": torch.full((count,), 3, dtype=torch.int64),
    }


def cameras(batch: int, scene_id: int = 3):
    return (torch.eye(4).repeat(batch, 1, 1).contiguous(), torch.eye(3).repeat(batch, 1, 1).contiguous(),
            torch.full((batch,), scene_id, dtype=torch.int64))


def service(**kwargs) -> tuple[RendererService, RecordingBackend]:
    backend = RecordingBackend()
    svc = RendererService(backend, height=3, width=4, max_views=4, allow_cpu_for_tests=True, **kwargs)
    svc.initialize(stage=None, device=CPU)
    svc.load_scene(3, **scene_kwargs())
    return svc, backend


def test_constructor_rejects_bad_arguments_with_reference_messages():
    backend = RecordingBackend()
    with pytest.raises(ValueError, match="height and width must be positive"):
        RendererService(backend, height=0, width=4)
    with pytest.raises(ValueError, match="render_every_n must be positive"):
        RendererService(backend, height=2, width=4, render_every_n=0)
    with pytest.raises(ValueError, match=r"Unsupported output name\(s\): bogus, normals\."):
        RendererService(backend, height=2, width=4, outputs=("rgb", "normals", "bogus"))


def test_calls_before_initialize_and_cpu_without_opt_in_are_refused():
    svc = RendererService(RecordingBackend(), height=2, width=2)
    with pytest.raises(RuntimeError, match=r"RendererService\.initialize\(stage, device\) must be called first"):
        svc.render(*cameras(1))
    with pytest.raises(ValueError, match="requires a CUDA device; got cpu"):
        svc.initialize(stage=None, device="cpu")


def test_registry_packs_offsets_in_registration_order():
    svc, backend = service()
    svc.load_scene(7, **scene_kwargs(5))
    assert backend.scenes == [(3, 0), (7, 2)]
    assert svc.registry.scene_ids == (3, 7)
    assert svc.registry.total_gaussians == 7
    assert svc.registry.offsets_tensor(device=CPU, require_cuda=False).tolist() == [0, 2, 7]
    with pytest.raises(ValueError, match="Scene 7 is already registered."):
        svc.load_scene(7, **scene_kwargs())
    with pytest.raises(ValueError, match="scene_offsets must be CUDA-resident."):
        svc.registry.offsets_tensor(device=CPU, require_cuda=True)


def test_scene_validation_names_the_first_bad_field():
    bad = scene_kwargs()
    bad["rotations"] = torch.ones((2, 3))
    with pytest.raises(ValueError, match="rotations dimension 1 must be 4; got 3."):
        GaussianScene(**bad).validate(device=CPU, require_cuda=False)
    bad = scene_kwargs()
    bad["semantic_ids"] = bad["semantic_ids"].int()
    with pytest.raises(ValueError, match="semantic_ids must have dtype torch.int64"):
        GaussianScene(**bad).validate(device=CPU, require_cuda=False)
    with pytest.raises(ValueError, match="must be CUDA-resident"):
        GaussianScene(**scene_kwargs()).validate(device=CPU, require_cuda=True)


def test_host_scene_id_checks():
    registry = SceneRegistry()
    registry.register(3, GaussianScene(**scene_kwargs()))
    registry.require_scene_ids(torch.tensor([3, 3]))
    with pytest.raises(ValueError, match=r"Unregistered scene ID\(s\): \[4, 9\]\."):
        registry.require_scene_ids(torch.tensor([9, 3, 4]))
    svc, _ = service()
    with pytest.raises(ValueError, match=r"Unregistered scene ID\(s\): \[5\]\."):
        svc.render(*cameras(2, scene_id=5))


def test_owned_outputs_start_at_the_inactive_contract_and_are_reused():
    svc, backend = service()
    first = svc.prepare_outputs(4)
    assert svc.prepare_outputs(4) is first
    assert torch.all(first["semantic_id"] == -1) and torch.all(first["rgb"] == 0)
    assert first["rgb"].shape == (4, 3, 4, 3) and first["semantic_id"].dtype == torch.int64
    with pytest.raises(ValueError, match="batch must be positive"):
        svc.prepare_outputs(0)
    with pytest.raises(ValueError, match="Batch has 5 cameras but service max_views is 4."):
        svc.prepare_outputs(5)
    out = svc.render(*cameras(4))
    assert out is first and torch.all(out["depth"] == 4.0)
    assert backend.calls.count("render") == 1


def test_render_cadence_replays_the_last_outputs():
    svc, backend = service(render_every_n=3)
    outputs = [svc.render(*cameras(2)) for _ in range(7)]
    assert backend.calls.count("render") == 3  # requests 1, 4 and 7
    assert all(o is outputs[0] for o in outputs)


def test_shutdown_releases_state_and_guards_later_calls():
    svc, backend = service()
    svc.prepare_outputs(2)
    svc.shutdown()
    assert backend.calls[-1] == "shutdown" and svc.workspace == {}
    with pytest.raises(RuntimeError, match="must be called first"):
        svc.synchronize()


def test_update_scene_transforms_checks_shapes():
    svc, backend = service()
    with pytest.raises(ValueError, match="scene_ids must have one entry per transform."):
        svc.update_scene_transforms(torch.tensor([3, 3]), torch.eye(4).repeat(3, 1, 1).contiguous())
    svc.update_scene_transforms(torch.tensor([3]), torch.eye(4)[None].contiguous())
    assert backend.calls[-1] == "update"


def lidar_kwargs(count: int = 3) -> dict[str, torch.Tensor]:
    return {
        "means": torch.zeros((count, 3)),
        "scales": torch.full((count, 3), 0.1),
        "rotations": torch.tensor([[1.0, 0.0, 0.0, 0.0]] * count),
        "opacities": torch.full((count,), 0.5),
        "semantic_ids": torch.arange(count, dtype=torch.int64),
    }


@pytest.mark.parametrize(
    "field,value,message",
    [
        ("means", torch.tensor([[float("nan"), 0.0, 0.0]] * 3), "means must be finite."),
        ("scales", torch.zeros((3, 3)), "scales must be finite and positive."),
        ("semantic_ids", torch.tensor([0, -1, 2]), "semantic_ids must be non-negative"),
        ("rotations", torch.tensor([[2.0, 0.0, 0.0, 0.0]] * 3), "rotations must be normalized WXYZ quaternions."),
        ("opacities", torch.tensor([0.5, 1.5, 0.5]), r"opacities must be finite and in \[0, 1\]."),
        ("reflectivity", torch.tensor([0.5, -0.5, 0.5]), r"reflectivity must be finite and in \[0, 1\]."),
    ],
)
def test_lidar_scene_value_rules(field, value, message):
    kwargs = lidar_kwargs()
    kwargs[field] = value
    with pytest.raises(ValueError, match=message):
        GaussianLidarScene(**kwargs).validate(device=CPU, require_cuda=False)


def test_lidar_registry_revisions_increase():
    registry = LidarSceneRegistry()
    scene = GaussianLidarScene(**lidar_kwargs(), revision=2)
    registry.register(17, scene)
    with pytest.raises(ValueError, match="LiDAR scene 17 is already registered."):
        registry.register(17, scene)
    with pytest.raises(ValueError, match="LiDAR scene 17 revision must increase from 2; got 2."):
        registry.revise(17, 2)
    revised = registry.revise(17, 5)
    assert revised.revision == 5 and revised.means is scene.means and registry.scene(17) is revised
    with pytest.raises(ValueError, match="Unregistered LiDAR scene ID: 4."):
        registry.scene(4)
    with pytest.raises(ValueError, match=r"Unregistered LiDAR scene ID\(s\): \[4\]\."):
        registry.require_scene_ids(torch.tensor([17, 4]))
    with pytest.raises(ValueError, match="Host LiDAR scene-ID validation accepts CPU tensors only."):
        registry.require_scene_ids(torch.empty(0, device="meta"))


def test_lidar_service_arguments():
    with pytest.raises(ValueError, match="max_sensors and max_rays must be positive."):
        GaussianLidarService(object(), max_sensors=0, max_rays=4)
    with pytest.raises(ValueError, match="returns must be exactly 1 or 2."):
        GaussianLidarService(object(), max_sensors=1, max_rays=4, returns=3)
    svc = GaussianLidarService(object(), max_sensors=1, max_rays=4)
    with pytest.raises(RuntimeError, match=r"GaussianLidarService\.initialize\(stage, device\) must be called first"):
        svc.load_scene(1, **lidar_kwargs())
