"""Generates h2_air_9sp.json from the reference's jet case inputs.

The 9-species / 19-reaction H2-air mechanism, its NASA-style thermo fits and the transport fits
ship with the reference as case files (cases/jet/Reaction.in, specie.in, viscosity.in,
conductivity.in, diffusion_coefficients.in). The GPU box has no copy of the reference, so this
script, run where the reference is mounted, turns them into one JSON data file that travels
with the package. Usage: python make_data.py /path/to/OpenCFD-Comb
"""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))
from ocfd_b200 import files  # noqa: E402


def main(ref):
    case = os.path.join(ref, "cases", "jet")
    sp = files.read_specie(os.path.join(case, "specie.in"))
    rc = files.read_reaction(os.path.join(case, "Reaction.in"))
    vis = files.read_fit_by_name(os.path.join(case, "viscosity.in"))
    cond = files.read_fit_by_name(os.path.join(case, "conductivity.in"))
    diff = files.read_diffusion(os.path.join(case, "diffusion_coefficients.in"))
    names = [s["name"] for s in sp["species"]]
    assert names == rc["species"], (names, rc["species"])
    out = dict(source="cases/jet of OpenCFD-Comb", thermo=sp, kinetics=rc,
               viscosity={n: vis[n] for n in names}, conductivity={n: cond[n] for n in names},
               diffusion=[[a, b, v] for (a, b), v in diff.items()])
    path = os.path.join(os.path.dirname(__file__), "h2_air_9sp.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", path, len(names), "species", rc["n_reac"], "reactions")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_data.py <path of the OpenCFD-Comb source tree (holds cases/jet)>")
    main(sys.argv[1])
