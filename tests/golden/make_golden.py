"""Writes the regression fixtures of tests/golden/ from the CPU oracle.

The reference ships no tests or golden outputs and cannot be compiled here, so
these fixtures are produced by the oracle (the C++ restatement in oracle/):
they pin the restatement against later changes and give the device path a
fixed target, they are not outputs of the reference itself.

    python tests/golden/make_golden.py     # from the repository root
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "amr-lbm-openmp-2d_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import numpy as np  # noqa: E402

import amrlbm  # noqa: E402

CASES = {
    # name: (params factory, time steps after start-up)
    "reference_default": (amrlbm.reference_params, 4),
    "small_16x16": (amrlbm.workload_small, 3),
}


def interior_digest(blocks, nx, ny):
    """sha256 over the interiors of h, g, C, P, Ux, Uy of the given blocks (each
    a dict of the reference-layout arrays), in the order given."""
    sha = hashlib.sha256()
    for b in blocks:
        for k in ("h", "g"):
            sha.update(np.ascontiguousarray(b[k][:, 1:nx + 1, 1:ny + 1], dtype="<f8").tobytes())
        sha.update(np.ascontiguousarray(b["C"][2:nx + 2, 2:ny + 2], dtype="<f8").tobytes())
        for k in ("P", "Ux", "Uy"):
            sha.update(np.ascontiguousarray(b[k], dtype="<f8").tobytes())
    return sha.hexdigest()


def snapshot(sim, p):
    leaves = [int(x) for x in sim.leaves()]
    topo = sim.topology()
    levels = np.bincount(np.asarray(topo["level"])[np.asarray(leaves) - 1],
                         minlength=p.max_levels + 1).tolist()
    out = sim.output()
    return {"counts": sim.counts(), "leaf_levels": levels, "leaves_sha256":
            hashlib.sha256(np.asarray(leaves, dtype="<i4").tobytes()).hexdigest(),
            "diag": {k: out[k] for k in ("mass", "rho_min", "rho_max", "u_max", "bubble_volume",
                                         "y_centroid", "rise_velocity", "phase_volume")},
            "fields_sha256": interior_digest([sim.download_block(b) for b in leaves],
                                             p.nx, p.ny)}


def main():
    from oracle_lib import Oracle
    for name, (factory, steps) in CASES.items():
        p = factory()
        orc = Oracle(p)
        orc.initialize_rising_bubble()
        rec = {"case": name, "steps": steps, "init": snapshot(orc, p)}
        orc.main_loop(steps)
        rec["after_steps"] = snapshot(orc, p)
        path = os.path.join(HERE, f"oracle_{name}.json")
        with open(path, "w") as f:
            json.dump(rec, f, indent=1, sort_keys=True)
            f.write("\n")
        print("wrote", path)


if __name__ == "__main__":
    main()
