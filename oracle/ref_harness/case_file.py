"""Case files of the reference-kernel harness (oracle/ref_harness/harness.cu).

Test and baseline infrastructure: the golden fixtures (tests/golden) and the
timing of the reference's own kernels beside the product (bench.py's baseline
leg) write their inputs with write_case.  The layout is the one harness.cu
documents: a CCCASE01 header, the scheme parameters, the species tables, the
boundary conditions, then per block its extents, processed-face records and
the geometry and state arrays of the ghosted box (i fastest).
"""
import struct

import numpy as np


def write_case(path, case):
    prm = case["params"]
    sp = prm.get("species")
    ns = 0 if sp is None else int(sp["n_spec"])
    with open(path, "wb") as f:
        f.write(b"CCCASE01")
        f.write(struct.pack("<8i", ns, len(case["blocks"]), prm["ngg"], prm["viscous_order"],
                            prm["reconstruction"], prm["limiter"], case["n_steps"], len(case["bcs"])))
        f.write(struct.pack("<3d", prm["prandtl_number"], prm["cfl"], prm["schmidt_number"]))
        if ns:
            for key in ("mw", "t_low", "t_mid", "t_high", "low_temp_coeff", "high_temp_coeff", "LJ_potent_inv",
                        "vis_coeff", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8"):
                f.write(np.ascontiguousarray(sp[key], dtype="<f8").tobytes())
        for bc in case["bcs"]:
            f.write(struct.pack("<4i", bc["label"], bc["kind"], bc.get("thermal_type", 0), 0))
            f.write(struct.pack("<7d", bc.get("t_wall", 300.0), bc.get("density", 0.0), bc.get("u", 0.0),
                                bc.get("v", 0.0), bc.get("w", 0.0), bc.get("pressure", 0.0),
                                bc.get("temperature", 0.0)))
            yk = np.zeros(ns)
            if "yk" in bc:
                yk[:] = np.asarray(bc["yk"])[:ns]
            f.write(yk.astype("<f8").tobytes())
        for b in case["blocks"]:
            f.write(struct.pack("<5i", *b["dims"], len(b["boundaries"]), len(b["inner_faces"])))
            for r in b["boundaries"]:
                f.write(struct.pack("<7i", *r))
            for r in b["inner_faces"]:
                f.write(struct.pack("<13i", *r))
            for key in ("jac", "metric", "bv", "yk"):
                f.write(np.ascontiguousarray(b[key], dtype="<f8").tobytes())
