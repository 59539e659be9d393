"""Generate tests/golden/reference_golden.json from the reference's own files.

Run once in a container that has the reference checkout; its path is the
required first argument (``python make_golden.py <reference checkout>``).  The GPU tests and the CPU suite
only read the committed JSON; nothing at test time reads the reference.

Pins extracted (all produced by the reference project itself):
  * notebooks/KitaevED.zip -> KitaevED.ipynb: the hard-coded 2x2 / 3x3
    honeycomb bond and hexagon lists and the recorded exact-diagonalisation
    outputs (E/N of the ground state, <W_p> of every hexagon);
  * test/test_lattice.cpp: nearest-neighbour lists of honeycomb(3);
  * test/test_derivative.cpp: seed, lattice, hidden size, weight std and the
    tolerances of the update-consistency and finite-difference tests.
"""
import ast
import json
import os
import re
import sys
import zipfile


def notebook_cells(ref):
    z = zipfile.ZipFile(os.path.join(ref, "notebooks", "KitaevED.zip"))
    nb = json.load(z.open("KitaevED.ipynb"))
    cells = []
    for c in nb["cells"]:
        if c["cell_type"] != "code":
            continue
        src = "".join(c["source"])
        outs = []
        for o in c.get("outputs", []):
            if "text" in o:
                outs.append("".join(o["text"]))
            elif "data" in o and "text/plain" in o["data"]:
                outs.append("".join(o["data"]["text/plain"]))
        cells.append((src, "\n".join(outs)))
    return cells


def literal_assign(src, name):
    m = re.search(r"^%s\s*=\s*(\[.*?^\])" % name, src, re.S | re.M)
    return ast.literal_eval(m.group(1))


def complex_lines(text):
    vals = []
    for line in text.strip().splitlines():
        vals.append(complex(line.strip()))
    return vals


def main(ref):
    cells = notebook_cells(ref)
    out = {"source": "dbucher97/rbm-nqs notebooks/KitaevED.zip, test/test_lattice.cpp, test/test_derivative.cpp"}
    for src, text in cells:
        for nm in ("bonds2", "plaqs2", "bonds3", "plaqs3"):
            if re.search(r"^%s\s*=" % nm, src, re.M):
                out[nm] = literal_assign(src, nm)
        if "ham2 = construct_operator" in src:
            out["ed_energy_per_site_2x2"] = complex_lines(text)[0].real
        if "ham3 = construct_operator" in src:
            out["ed_energy_per_site_3x3"] = complex_lines(text)[0].real
        if "for plaq in plaqs2" in src:
            out["ed_wp_2x2"] = [v.real for v in complex_lines(text)]
        if "for plaq in plaqs3" in src:
            out["ed_wp_3x3"] = [v.real for v in complex_lines(text)]

    lat = open(os.path.join(ref, "test", "test_lattice.cpp")).read()
    nns = {}
    for site, vals in re.findall(r"nns_at(\d+)_should = \{([0-9, ]+)\}", lat):
        nns[site] = [int(v) for v in vals.split(",")]
    out["honeycomb3_nns"] = nns

    der = open(os.path.join(ref, "test", "test_derivative.cpp")).read()
    out["test_derivative"] = {
        "seed": int(re.search(r"#define SEED (\d+)", der).group(1)),
        "lattice": "honeycomb(5)",
        "n_hidden": 10,
        "weight_std": 0.2,
        "theta_update_tol": 1e-15,
        "rbm_fd_tol_per_param": 1e-15,
        "rbm_fd_dw_scale": 1e-7,
        "pf_inv_drift_tol": 1e-10,
        "pf_pfaffian_drift_tol": 1e-12,
        "pf_fd_tol_per_param": 1e-14,
        "pf_fd_dw_scale": 1e-8,
        "pf_weight_std": 0.1,
        "n_updates": 100,
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the rbm-nqs reference checkout>")
    main(sys.argv[1])
