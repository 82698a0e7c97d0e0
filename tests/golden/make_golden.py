"""Golden fixtures: the reference's own kernels on small cases.

Step 1 (here, no GPU):   python tests/golden/make_golden.py write-cases DIR
    writes DIR/<case>.bin in the case layout read by oracle/ref_harness/harness.cu
Step 2 (on a B200):      for c in DIR/*.bin: oracle/_ref/ref_harness_{ms,air} c c.out
    runs the reference's kernels (built from the reference sources by
    oracle/ref_harness/build_ref.sh) for n steady explicit-Euler steps
Step 3 (here):           python tests/golden/make_golden.py pack DIR
    packs inputs and the reference's outputs into tests/golden/<case>.npz

Each case is a small seeded input of the synthetic species set (see
combustioncodegpu_b200/cases.py); together they cover the air and the
9-species models, inviscid and viscous fluxes, MUSCL and first-order
reconstruction, outflow, inflow, isothermal and adiabatic walls, periodic
faces and a two-block interface.
"""
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from combustioncodegpu_b200 import cases  # noqa: E402
from oracle.ref_harness.case_file import write_case  # noqa: E402,F401

HERE = os.path.dirname(os.path.abspath(__file__))


def golden_cases():
    sp = cases.synthetic_species()
    out = {}
    c = cases.case_sod(20, 5, 5)
    c["n_steps"] = 4
    out["sod_air"] = c
    c = cases.case_box(8, species=sp, seed=11)
    c["n_steps"] = 3
    out["box_ms"] = c
    c = cases.case_channel((9, 6, 5), species=sp, seed=12)
    c["n_steps"] = 3
    out["channel_ms"] = c
    c = cases.case_multiblock(([6, 7], [6], [5]), species=sp, seed=13)
    c["n_steps"] = 2
    out["multiblock_ms"] = c
    # viscous air (Sutherland) with first-order reconstruction
    dims = (7, 6, 5)
    jac, met = cases.make_block(dims, (1e-3, 0.8e-3, 0.6e-3))
    rng = np.random.default_rng(14)
    ng = (dims[0] + 4) * (dims[1] + 4) * (dims[2] + 4)
    T = 300 + 200 * rng.random(ng)
    p = 101325 * (1 + 0.02 * rng.standard_normal(ng))
    rho = p * cases.MW_AIR / (cases.R_U * T)
    u, v, w = (30 * rng.standard_normal(ng) for _ in range(3))
    faces = []
    for a in range(3):
        faces += cases.periodic_raw(dims, a)
    prm = cases.default_params(None, viscous=True)
    prm["reconstruction"] = 1
    out["air_visc_o1"] = {"name": "air_visc_o1", "params": prm, "bcs": [], "n_steps": 3,
                          "blocks": [{"dims": dims, "jac": jac, "metric": met,
                                      "bv": np.stack([rho, u, v, w, p, T]), "yk": np.zeros((0, ng)),
                                      "boundaries": [], "inner_faces": faces}]}
    return out


def read_case(path):
    """Inverse of write_case: the case dict exactly as the harness read it."""
    data = open(path, "rb").read()
    assert data[:8] == b"CCCASE01", path
    pos = 8

    def take(fmt, n):
        nonlocal pos
        v = np.frombuffer(data, fmt, n, pos).copy()
        pos += v.itemsize * n
        return v

    ns, nb, ngg, visc, rec, lim, n_steps, n_bc = (int(v) for v in take("<i4", 8))
    Pr, cfl, Sc = (float(v) for v in take("<f8", 3))
    prm = {"inviscid_scheme": 3, "reconstruction": rec, "limiter": lim, "viscous_order": visc, "ngg": ngg,
           "cfl": cfl, "prandtl_number": Pr, "schmidt_number": Sc, "species": None}
    if ns:
        sp = {"n_spec": ns}
        for key, n in (("mw", ns), ("t_low", ns), ("t_mid", ns), ("t_high", ns), ("low_temp_coeff", 7 * ns),
                       ("high_temp_coeff", 7 * ns), ("LJ_potent_inv", ns), ("vis_coeff", ns),
                       ("WjDivWi_to_One4th", ns * ns), ("sqrt_WiDivWjPl1Mul8", ns * ns)):
            sp[key] = take("<f8", n)
        for key in ("low_temp_coeff", "high_temp_coeff"):
            sp[key] = sp[key].reshape(ns, 7)
        for key in ("WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8"):
            sp[key] = sp[key].reshape(ns, ns)
        prm["species"] = sp
    bcs = []
    for _ in range(n_bc):
        label, kind, tt, _pad = (int(v) for v in take("<i4", 4))
        t_wall, rho, u, v, w, p, T = (float(x) for x in take("<f8", 7))
        yk = take("<f8", ns)
        bcs.append({"label": label, "kind": kind, "thermal_type": tt, "t_wall": t_wall, "density": rho, "u": u,
                    "v": v, "w": w, "pressure": p, "temperature": T, "yk": yk})
    blocks = []
    for _ in range(nb):
        mx, my, mz, n_bnd, n_in = (int(v) for v in take("<i4", 5))
        bnd = [list(map(int, take("<i4", 7))) for _ in range(n_bnd)]
        inf = [list(map(int, take("<i4", 13))) for _ in range(n_in)]
        ng = (mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg)
        jac = take("<f8", ng)
        met = take("<f8", 9 * ng).reshape(9, ng)
        bv = take("<f8", 6 * ng).reshape(6, ng)
        yk = take("<f8", ns * ng).reshape(ns, ng)
        blocks.append({"dims": (mx, my, mz), "boundaries": bnd, "inner_faces": inf, "jac": jac, "metric": met,
                       "bv": bv, "yk": yk})
    assert pos == len(data)
    return {"params": prm, "bcs": bcs, "blocks": blocks, "n_steps": n_steps}


def read_output(path, case):
    sp = case["params"].get("species")
    ns = 0 if sp is None else int(sp["n_spec"])
    nv = 5 + ns
    data = open(path, "rb").read()
    assert data[:8] == b"CCOUT001", path
    pos = 8

    def ints(n):
        nonlocal pos
        v = np.frombuffer(data, "<i4", n, pos)
        pos += 4 * n
        return v.copy()

    def dbl(n):
        nonlocal pos
        v = np.frombuffer(data, "<f8", n, pos)
        pos += 8 * n
        return v.copy()

    nb = int(ints(1)[0])
    out = {}
    for b, blk in enumerate(case["blocks"]):
        mx, my, mz = blk["dims"]
        ng = (mx + 4) * (my + 4) * (mz + 4)
        n = mx * my * mz
        nbd = int(ints(1)[0])
        out["b%d_boundaries" % b] = ints(9 * nbd).reshape(nbd, 9)
        nin = int(ints(1)[0])
        out["b%d_inner_faces" % b] = ints(26 * nin).reshape(nin, 26)
        out["b%d_dq1" % b] = dbl(nv * n).reshape(nv, n)
        out["b%d_dt1" % b] = dbl(n)
        out["b%d_bv" % b] = dbl(6 * ng).reshape(6, ng)
        if ns:
            out["b%d_yk" % b] = dbl(ns * ng).reshape(ns, ng)
        out["b%d_cv" % b] = dbl(nv * ng).reshape(nv, ng)
        out["b%d_mul" % b] = dbl(ng)
        out["b%d_cond" % b] = dbl(ng)
        if ns:
            out["b%d_rho_d" % b] = dbl(ns * ng).reshape(ns, ng)
    out["residual"] = dbl(4)
    assert nb == len(case["blocks"]) and pos == len(data), (path, pos, len(data))
    return out


def pack(case, ref):
    """Inputs and reference outputs of one case as one npz dict."""
    prm = case["params"]
    sp = prm.get("species")
    d = {"n_steps": case["n_steps"], "n_block": len(case["blocks"])}
    for k in ("inviscid_scheme", "reconstruction", "limiter", "viscous_order", "ngg", "cfl", "prandtl_number",
              "schmidt_number"):
        d["param_" + k] = prm[k]
    if sp is not None:
        for k in ("n_spec", "mw", "t_low", "t_mid", "t_high", "low_temp_coeff", "high_temp_coeff",
                  "LJ_potent_inv", "vis_coeff", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8"):
            d["species_" + k] = np.asarray(sp[k])
    d["n_bc"] = len(case["bcs"])
    for i, bc in enumerate(case["bcs"]):
        for k, v in bc.items():
            d["bc%d_%s" % (i, k)] = np.asarray(v)
    for b, blk in enumerate(case["blocks"]):
        d["b%d_dims" % b] = np.asarray(blk["dims"])
        d["b%d_raw_boundaries" % b] = np.asarray(blk["boundaries"], dtype=np.int32).reshape(-1, 7)
        d["b%d_raw_inner_faces" % b] = np.asarray(blk["inner_faces"], dtype=np.int32).reshape(-1, 13)
        for k in ("jac", "metric", "bv", "yk"):
            d["b%d_in_%s" % (b, k)] = np.asarray(blk[k])
    for k, v in ref.items():
        d["ref_" + k] = v
    return d


def load(name):
    """Case dict (cases.py format) and reference outputs of a packed fixture."""
    z = np.load(os.path.join(HERE, name + ".npz"))
    prm = {k[len("param_"):]: z[k].item() for k in z.files if k.startswith("param_")}
    if "species_n_spec" in z.files:
        sp = {k[len("species_"):]: z[k] for k in z.files if k.startswith("species_")}
        sp["n_spec"] = int(sp["n_spec"])
        prm["species"] = sp
    else:
        prm["species"] = None
    bcs = []
    for i in range(int(z["n_bc"])):
        pre = "bc%d_" % i
        bc = {}
        for k in z.files:
            if k.startswith(pre):
                v = z[k]
                bc[k[len(pre):]] = v.item() if v.ndim == 0 else v
        bcs.append(bc)
    blocks = []
    for b in range(int(z["n_block"])):
        blocks.append({
            "dims": tuple(int(v) for v in z["b%d_dims" % b]),
            "boundaries": [list(map(int, r)) for r in z["b%d_raw_boundaries" % b]],
            "inner_faces": [list(map(int, r)) for r in z["b%d_raw_inner_faces" % b]],
            "jac": z["b%d_in_jac" % b], "metric": z["b%d_in_metric" % b], "bv": z["b%d_in_bv" % b],
            "yk": z["b%d_in_yk" % b],
        })
    case = {"name": name, "params": prm, "bcs": bcs, "blocks": blocks, "n_steps": int(z["n_steps"])}
    ref = {k[len("ref_"):]: z[k] for k in z.files if k.startswith("ref_")}
    return case, ref


NAMES = ["sod_air", "box_ms", "channel_ms", "multiblock_ms", "air_visc_o1"]


def main():
    cmd, d = sys.argv[1], sys.argv[2]
    cs = golden_cases()
    if cmd == "write-cases":
        os.makedirs(d, exist_ok=True)
        for name, c in cs.items():
            ms = c["params"].get("species") is not None
            write_case(os.path.join(d, "%s.%s.bin" % (name, "ms" if ms else "air")), c)
        print("wrote", sorted(os.listdir(d)))
    elif cmd == "pack":
        for name, c0 in cs.items():
            ms = c0["params"].get("species") is not None
            fn = os.path.join(d, "%s.%s.bin" % (name, "ms" if ms else "air"))
            c = read_case(fn)
            ref = read_output(fn + ".out", c)
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **pack(c, ref))
            print("packed", name)


if __name__ == "__main__":
    main()
