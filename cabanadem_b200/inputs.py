"""Flat JSON configuration, mirroring ``CabanaDEM::Inputs`` (src/CabanaDEM_Input.hpp:41-82).

Schema: ``{"key": {"value": v, "unit"|"units": u}, ...}``.  The constructor adds
``num_steps = int(final_time / timestep)`` (Input.hpp:50-54); the reference's solver
loop then runs ``num_steps + 1`` steps (src/CabanaDEM_Solver.hpp:79).
"""
from __future__ import annotations

import json


def splitString(s: str, delimiter: str):
    """src/CabanaDEM_Input.hpp:24-38: split on every delimiter, keep empty fields."""
    return s.split(delimiter)


class Inputs:
    def __init__(self, source):
        if isinstance(source, dict):
            self.inputs = json.loads(json.dumps(source))
        else:
            with open(source) as f:
                self.inputs = json.load(f)
        tf = float(self.inputs["final_time"]["value"])
        dt = float(self.inputs["timestep"]["value"])
        self.inputs["num_steps"] = {"value": int(tf / dt)}

    def __getitem__(self, label):
        return self.inputs[label]["value"]

    def units(self, label):
        entry = self.inputs[label]
        return entry["units"] if "units" in entry else ""

    def contains(self, label):
        return label in self.inputs
