"""Driver with the reference's command line and loop (run_simulation.py:16-77):

    python -m dimcv_sph_b200.run_simulation --scene_file scene.json

Writes a PNG frame to result_images/ every output interval, and a PLY frame
to result_ply/ when the scene sets "exportPLY", clearing both folders first.
`--max_steps` bounds the run; a file named `stop` in the working directory
ends it, as in the reference.
"""
from __future__ import annotations

import argparse
import os
import shutil
import time
from pathlib import Path

from .config_builder import SimConfig
from .particle_system import ParticleSystem


def main(argv=None):
    parser = argparse.ArgumentParser(description="Dynamic Importance Monte Carlo Vortical SPH (B200)")
    parser.add_argument("--scene_file", default="", help="scene file")
    parser.add_argument("--max_steps", type=int, default=None, help="stop after this many steps")
    parser.add_argument("--device", default="cuda")
    args = parser.parse_args(argv)
    image_path = Path("result_images")  # run_simulation.py:18-27
    if image_path.exists():
        shutil.rmtree(image_path)
    image_path.mkdir(parents=True, exist_ok=True)
    config = SimConfig(scene_file_path=args.scene_file)
    export_ply = bool(config.get_cfg("exportPLY") or False)
    ply_path = None
    if export_ply:
        ply_path = Path("result_ply")
        if ply_path.exists():
            shutil.rmtree(ply_path)
        ply_path.mkdir(parents=True, exist_ok=True)
    simulation_time = config.get_cfg("simulationTime")
    substeps = config.get_cfg("numberOfStepsPerRenderUpdate") or 1
    output_interval = max(1, int(0.016 / config.get_cfg("timeStepSize")))

    ps = ParticleSystem(config, GGUI=False, device=args.device, verbose=True)
    solver = ps.build_solver()
    solver.initialize()

    cnt = cnt_output = 0
    t = 0.0
    t0 = time.time()
    while True:
        for _ in range(substeps):
            solver.step()
        cnt += 1
        t += solver.dt[None]
        if cnt % output_interval == 0:
            solver.export_png(cnt_output, image_path)
            if export_ply:
                solver.export_ply(cnt_output, ply_path)
            cnt_output += 1
        if cnt % 50 == 0:
            print(f"Simulation Time = {t:.2f}s")
            print("Fluid_particle_num = {}".format(solver.ps.fluid_particle_num[None]))
            print("Sample_num = ", solver.num_samples[None])
            print(f"wall {time.time() - t0:.1f}s")
        if t > simulation_time or os.path.exists("stop") or (args.max_steps and cnt >= args.max_steps):
            break
    solver.flush_exports()  # PLY frames are written asynchronously
    return solver


if __name__ == "__main__":
    main()
