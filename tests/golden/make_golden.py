"""Extract the reference's own printed run output from its example notebook.

Reads RobertRyne/OpenSpaceCharge examples/benchmark.ipynb (the reference checkout must be
present at REF, default /root/reference) and writes notebook_runs.json: for each run of
test_opensc saved in the notebook, the namelist grid, the particle bounding box printed by
gendist, and the mesh min/max/delta printed after get_mesh_quantities
(code/test_opensc.f90:151-154), plus the published cathode cross-method differences
(examples/benchmark.ipynb cells 25-26).  The JSON is committed; tests never read REF.
"""
import json
import os
import re
import sys

REF = os.environ.get("OPENSC_REF", "/root/reference")
NB = os.path.join(REF, "examples", "benchmark.ipynb")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "notebook_runs.json")


def floats(line):
    return [float(v) for v in re.findall(r"[-+]?\d+\.\d+E[-+]\d+|[-+]?\d+\.\d+", line)]


def main():
    nb = json.load(open(NB))
    runs = []
    for idx, cell in enumerate(nb["cells"]):
        if cell["cell_type"] != "code":
            continue
        for o in cell.get("outputs", []):
            txt = "".join(o.get("text", []))
            if "mesh xmin,xmax" not in txt:
                continue
            g = {}
            for key in ("NXHI", "NYHI", "NZHI", "NXLO", "NYLO", "NZLO"):
                m = re.search(key + r"=\s*(\d+)", txt)
                g[key.lower()] = int(m.group(1))
            run = {"cell": idx, "grid": g}
            for tag in ("particle xmin,xmax", "particle ymin,ymax", "particle zmin,zmax",
                        "mesh xmin,xmax", "mesh ymin,ymax", "mesh zmin,zmax", "delta(1:3)"):
                line = [l for l in txt.splitlines() if tag in l][0]
                run[tag] = floats(line.split("=", 1)[1])
            m = re.search(r"Time for space charge calc \(s\):\s*([0-9.Ee+-]+)", txt)
            run["cpu_time_s"] = float(m.group(1)) if m else None
            runs.append(run)
    cross = {}
    for idx in (25, 26):
        cell = nb["cells"][idx]
        src = "".join(cell["source"])
        val = float("".join(cell["outputs"][0]["data"]["text/plain"]))
        cross["3v1" if "3 vs 1" in src else "2v1"] = {"cell": idx, "max_rel_Ez_diff": val}
    json.dump({"source": "examples/benchmark.ipynb", "runs": runs, "cathode_cross_method": cross},
              open(OUT, "w"), indent=1)
    print(OUT, len(runs), "runs")


if __name__ == "__main__":
    sys.exit(main())
