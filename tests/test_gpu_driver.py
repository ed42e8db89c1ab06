"""The reference's driver loop (run_simulation.py:15-77) on the small channel
scene written to a JSON file: one output interval (0.016 s / dt steps) gives
one PNG frame in result_images/ and, with exportPLY, one PLY in result_ply/."""
import json

import pytest

from dimcv_sph_b200 import scenes

pytestmark = pytest.mark.gpu


def test_driver_writes_frames(cuda, tmp_path, monkeypatch):
    from dimcv_sph_b200 import run_simulation
    cfg = scenes.channel2d(trim_cylinder=True).config
    cfg["Configuration"]["exportPLY"] = True
    scene = tmp_path / "scene.json"
    scene.write_text(json.dumps(cfg))
    monkeypatch.chdir(tmp_path)
    (tmp_path / "result_images").mkdir()
    (tmp_path / "result_images" / "old.png").write_bytes(b"stale")
    steps = int(0.016 / cfg["Configuration"]["timeStepSize"])
    solver = run_simulation.main(["--scene_file", str(scene), "--max_steps", str(steps)])
    assert solver.cnt == steps
    assert sorted(p.name for p in (tmp_path / "result_images").iterdir()) == ["vorticity_0000.png"]
    assert sorted(p.name for p in (tmp_path / "result_ply").iterdir()) == ["frame_0000.ply"]
