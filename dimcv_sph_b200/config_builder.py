"""Scene configuration reader with the reference's interface
(config_builder.py:3-41): `get_cfg(name)` returns None for a missing key of
the "Configuration" object; the block accessors return [] when absent.
A SimConfig can also be built from a dict (scene builders use that)."""
from __future__ import annotations

import copy
import json


class SimConfig:
    def __init__(self, scene_file_path=None, config: dict | None = None, verbose: bool = False) -> None:
        if config is not None:
            self.config = copy.deepcopy(config)
        else:
            with open(scene_file_path, "r") as f:
                self.config = json.load(f)
        if verbose:
            print(self.config)

    def get_cfg(self, name, enforce_exist=False):
        section = self.config.get("Configuration", {})
        if name not in section:
            if enforce_exist:
                raise KeyError(f"missing configuration key {name!r}")
            return None
        return section[name]

    def _list(self, key):
        return self.config.get(key, [])

    def get_rigid_bodies(self):
        return self._list("RigidBodies")

    def get_rigid_blocks(self):
        return self._list("RigidBlocks")

    def get_fluid_blocks(self):
        return self._list("FluidBlocks")

    def get_fluid_emitters(self):
        return self._list("FluidEmitters")
