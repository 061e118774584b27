"""Generates the committed oracle fixtures in this folder.

    python tests/golden/make_golden.py

The fixture is a regression pin of the oracle on one small seeded case
(Si8, 20 Ry, 24^3 grid, 6 CP steps with moving atoms): the G-set hash, the
energies of every step, the ORTHO_X iteration counts and the first forces.
It is produced by the oracle itself (the reference cannot be run here), so it
guards the restatement against regressions; it is not an external pin.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "cp-paw_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def run_case(binding, nsteps: int = 6) -> dict:
    from cuwaves import systems

    s = systems.si_cell(1, grid=(24, 24, 24), epw_psi_ry=20.0, name="Si8-20Ry")
    inp = systems.build_inputs(s)
    w = binding.open_oracle(inp).setup().initialize()
    res = {"ngl": int(inp["ngl"]),
           "igvec_sha256": hashlib.sha256(inp["igvec"].astype("<i4").tobytes()).hexdigest(),
           "etot": [], "ekin": [], "ekinpsi": [], "iters": []}
    for k in range(nsteps):
        out, f = w.cp_step(move_atoms=True)
        res["etot"].append(float(out[0]))
        res["ekin"].append(float(out[1]))
        res["ekinpsi"].append(float(out[2]))
        res["iters"].append(int(out[4]))
        if k == 0:
            res["force0"] = f.tolist()
    w.close()
    return res


if __name__ == "__main__":
    import binding

    binding.build()
    out = run_case(binding)
    with open(os.path.join(HERE, "oracle_si8_20ry.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", os.path.join(HERE, "oracle_si8_20ry.json"))
