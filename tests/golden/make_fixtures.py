"""Regenerate the committed golden fixtures from the reference checkout.

Run in a container that has the reference mounted (default /root/reference):

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

Outputs (committed, read by the tests; nothing reads the reference at test time):
  * research_*.request.json - the reference's shipped example requests
    (examples/research_{slump,hydrostatic_water,coupled_patch}.yaml) as JSON;
  * reference_values.json   - the reference's own published FP64 results for those
    requests and its known-answer constants, each with the file:line it is quoted from.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import yaml

HERE = Path(__file__).resolve().parent

EXAMPLES = ["research_slump", "research_hydrostatic_water", "research_coupled_patch"]

# Published values (FP64 reference runs of the examples above), quoted verbatim.
REFERENCE_VALUES = {
    "research_hydrostatic_water": {
        "source": "docs/validation.md:232-236 (signed channel, new residual); docs/validation.md:153-157",
        "observables": {
            "wall_normal_traction_energy_j": 1.0219846729e-8,
            "energy_residual_j": 1.4254529794e-6,
            "hydrostatic_max_relative_error": 0.0115138566,
            "hydrostatic_rms_relative_error": 0.0034430221,
            "mass_residual_kg": -8.673617379884035e-19,
            "momentum_residual_kg_m_s": 4.770490026058286e-18,
            "rejected_steps": 0.0,
            "limited_steps": 0.0,
        },
        "digits": 10,
    },
    "research_slump": {
        "source": "docs/validation.md:232-236",
        "observables": {
            "wall_normal_traction_energy_j": -9.7731734973e-6,
            "energy_residual_j": 7.3769595864e-5,
        },
        "digits": 10,
    },
    "research_coupled_patch": {
        "source": "docs/validation.md:232-236",
        "observables": {
            "wall_normal_traction_energy_j": -3.4963973432e-6,
            "energy_residual_j": -7.1239144793e-6,
        },
        "digits": 10,
    },
    "known_answers": {
        "paste_return": {
            "source": "core/tests/formal_examples.rs:11-25; tests/test_formal.py:73-92",
            "material_shear_rheology": [1000.0, 1000.0, 0.2, 30.0, 10.0, 0.6],
            "trial_equivalent_stress": 80.0,
            "dt": 0.0014,
            "equivalent_stress": 78.0059568837,
            "equivalent_stress_tol": 1e-9,
            "plastic_increment": 0.001595234493,
            "plastic_increment_tol": 1e-12,
        },
        "water_eos": {
            "source": "core/tests/formal_examples.rs:27-44",
            "material_liquid": [1000.0, 1e5, 0.2, 1e-3],
            "depth": 0.01,
            "gravity": 9.81,
            "pressure": 98.186663,
            "pressure_tol": 5e-7,
            "volume_ratio_after": 0.997,
        },
        "pellet": {
            "source": "tests/test_formal.py:62-69",
            "mass_grams": 0.3732212072464674,
        },
        "pashias": {
            "source": "core/src/mpm/fixtures.rs:723-736",
            "tau_prime": 0.1,
        },
    },
}


def main(reference_root: str = "/root/reference") -> None:
    root = Path(reference_root)
    for name in EXAMPLES:
        req = yaml.safe_load((root / "examples" / f"{name}.yaml").read_text())
        (HERE / f"{name}.request.json").write_text(json.dumps(req, indent=1, sort_keys=True) + "\n")
    (HERE / "reference_values.json").write_text(json.dumps(REFERENCE_VALUES, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main(*sys.argv[1:])
