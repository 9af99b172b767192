"""Golden profiles from the reference's own profile generator, set_background_profiles.ipynb.

Run in the build container (where the reference is mounted read-only):

    python tests/golden/notebook/make_notebook_golden.py /root/reference/set_background_profiles.ipynb

It executes the notebook's numeric code cells (N^2(t), the stretched grid, the stretching
matrix, the first baroclinic mode, the ocean-Charney profile, u_bar, S) with its own settings
(nz = 32, alpha = 1), skipping the plotting cells, in a temporary directory where the notebook's
last cell writes S.dat, H.dat, zc.dat and UBar.dat.  It stores those four files' values and
the deformation radii that the notebook's cell 9 printed when it was saved (its stored output,
read as text) in notebook_profiles_nz32.npz next to this script.  tests/test_oracle.py checks
inputs.notebook_profiles and the stretching-matrix eigenvalues against them.
"""
import json
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(path):
    nb = json.load(open(path))
    cells = [c for c in nb["cells"] if c["cell_type"] == "code"]
    src = ["".join(c["source"]) for c in cells]
    # the cells that compute (no matplotlib): imports, settings, N2, grid, L, modes, oc profile,
    # u_bar, S, and the cell that writes the .dat files
    keep = []
    printed = None
    for s, c in zip(src, cells):
        if "print(H_tot*np.sort(1/np.sqrt(-vals))/1E3)" in s:
            printed = "".join("".join(o.get("text", "")) for o in c.get("outputs", []) if o.get("name") == "stdout")
            continue
        if "plt." in s or "matplotlib" in s:
            lines = [ln for ln in s.split("\n") if "matplotlib" not in ln and "plt" not in ln]
            s = "\n".join(lines)
            if not s.strip() or "subplots" in "".join(c["source"]):
                continue
        keep.append(s)
    radii = [float(x) if x != "nan" else np.nan for x in re.findall(r"nan|[-+]?\d+\.\d+(?:[eE][-+]?\d+)?",
                                                                       printed.split("\n\n")[0])]
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            env = {}
            for s in keep:
                exec(compile(s, "<notebook>", "exec"), env)
            vals = {k: np.fromfile(os.path.join(d, f"{k}.dat")) for k in ("S", "H", "zc", "UBar")}
        finally:
            os.chdir(cwd)
    out = os.path.join(HERE, "notebook_profiles_nz32.npz")
    np.savez(out, radii_printed=np.array(radii), nz=env["nz"], alpha=env["alpha"], H_tot=env["H_tot"], **vals)
    print("wrote", out, {k: v.shape for k, v in vals.items()}, len(radii), "printed radii")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/set_background_profiles.ipynb")
