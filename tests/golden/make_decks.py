"""Writes the reference's regression input decks as test fixtures.

The FerroX tree ships inputs decks for its regression runs
(Exec/regression_inputs/3D_MFIM/inputs_mfim_Noeb and
Exec/regression_inputs/MIS/input_mis) and examples with an embedded metal
boundary (Exec/Examples/inputs_mfim_eb, inputs_mfis_eb), but no outputs.  The parity tests run
these decks through both the GPU library and the CPU oracle; the reference
tree is not present where the GPU tests run, so the decks travel as fixtures.
This script keeps each `key = value` line (comments and blank lines dropped,
values as written) and is run by hand where the reference tree exists:

    python tests/golden/make_decks.py /path/to/FerroX
"""
from __future__ import annotations

import os
import sys

DECKS = {
    "3D_MFIM_inputs_mfim_Noeb.inputs": "Exec/regression_inputs/3D_MFIM/inputs_mfim_Noeb",
    "MIS_input_mis.inputs": "Exec/regression_inputs/MIS/input_mis",
    "Examples_inputs_mfim_eb.inputs": "Exec/Examples/inputs_mfim_eb",
    "Examples_inputs_mfis_eb.inputs": "Exec/Examples/inputs_mfis_eb",
}


def strip(text: str) -> str:
    out = []
    for line in text.splitlines():
        line = line.split("#", 1)[0].rstrip()
        if line.strip():
            out.append(line.strip())
    return "\n".join(out) + "\n"


def main(root: str) -> None:
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "decks")
    os.makedirs(here, exist_ok=True)
    for name, rel in DECKS.items():
        with open(os.path.join(root, rel)) as f:
            text = strip(f.read())
        with open(os.path.join(here, name), "w") as f:
            f.write(f"# from FerroX {rel} (comments dropped)\n" + text)
        print(name)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
