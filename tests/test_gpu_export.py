"""Frame export of the channel after a few steps: the ASCII PLY of
karman_vortex.py:122-214 (header, one row per active particle: x y z, the
vorticity, colour, object id and particle type) and the PNG of :38-121.
PLY frames are written asynchronously; the file of a frame must hold the
state of the step it was submitted after, even when later steps run before
it is written."""
import numpy as np
import pytest

from dimcv_sph_b200 import scenes

pytestmark = pytest.mark.gpu


def test_ply_and_png_frames(cuda, tmp_path):
    from dimcv_sph_b200.particle_system import ParticleSystem
    ps = ParticleSystem(scenes.channel2d(trim_cylinder=True))
    solver = ps.build_solver()
    solver.initialize()
    for _ in range(3):
        solver.step()
    n = int(ps.is_active[: ps.particle_num[None]].sum().item())
    from dimcv_sph_b200.export import _object_sets, format_ply
    m = ps.particle_num[None]
    expect = format_ply(solver.x_temp[:m].cpu().numpy(), ps.vorticity[:m].cpu().numpy(),
                        ps.color[:m].cpu().numpy(), ps.object_id[:m].cpu().numpy(),
                        ps.is_active[:m].cpu().numpy(), _object_sets(ps))
    ply = solver.export_ply(7, tmp_path / "ply")
    assert ply.name == "frame_0007.ply"
    solver.step()  # runs while the frame is copied and written
    solver.step()
    solver.flush_exports()
    assert ply.read_text() == expect
    text = ply.read_text().splitlines()
    end = text.index("end_header")
    assert text[0] == "ply" and text[2] == f"element vertex {n}"
    rows = text[end + 1:]
    assert len(rows) == n
    cols = np.array([r.split() for r in rows])
    assert cols.shape[1] == 11
    xyz = cols[:, :3].astype(np.float64)
    assert np.all(xyz[:, 2] == 0.0) and np.all((xyz[:, 0] >= 0) & (xyz[:, 0] <= 4))
    ptype = cols[:, 10].astype(int)
    assert set(ptype) <= {0, 1, 2, 3, 4} and {0, 2} <= set(ptype)  # fluid block and rigid blocks present
    png = solver.export_png(7, tmp_path / "png")
    assert png.name == "vorticity_0007.png" and png.read_bytes()[:8] == b"\x89PNG\r\n\x1a\n"
    from PIL import Image
    a = np.asarray(Image.open(png))
    assert a.shape == (512, 2048, 4) and (a[..., 3] > 0).sum() > 1000
