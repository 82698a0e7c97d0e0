"""The reference's input files: readers (and writers) for the data formats on
either side of the residual path.

A reference case directory `input_files/` holds
  grid/grid   0.grd                       block sizes and coordinates (Mesh.cpp:566-614)
  boundary_condition/boundary   0.txt     boundary faces per block (Mesh.cpp:616-636)
  boundary_condition/inner   0.txt        block interfaces (Mesh.cpp:638-670)
  setup/{0,1,2,3,4,9}_*.txt               "type key = value" parameters (Parameter.cpp:44-71)
  setup/5_boundary_condition.txt          condition type, name and label (BoundCond.cu:315-409)
  setup/6_inflow.txt, setup/7_wall.txt    per-label inflow / wall values (BoundCond.cpp:10-137)
  setup/8_initialization.txt              initial state from inflow labels (Initialize.cu:24-120)
  <mechanism_file>, <therm_file>, <tran_file>   ChemData format (ChemData.cpp:10-261)

load_case() turns such a directory into the case dict that Driver.from_case
takes: the ghost grid is built as Mesh::init_ghost_grid does (Mesh.cpp:718-
923: reflection across the block faces, interface ghosts from the neighbour
block, parallelogram edges and corners), metrics by Block::compute_jac_metric
(cases.jac_metric), faces registered by the library (cc_register_*).
write_case() writes a case dict in the same formats (used to run the
synthetic workloads through the readers, and to hand them to the reference).
Single-process files only (the "   0" suffix); MPI parallel faces are not read.
"""
import os

import numpy as np

from . import cases

SETUP_FILES = ["0_global_control.txt", "1_grid_information.txt", "2_scheme.txt", "3_species_reactions.txt",
               "4_laminar_turbulent.txt", "9_transport_property.txt"]
BC_KIND = {"wall": 2, "inflow": 5, "outflow": 6}


# ------------------------------------------------------------- parameters

def read_parameters(setup_dir):
    """All "int/double/bool/string key = value" lines of the setup files
    (Parameter.cpp:44-71); first definition wins, as with std::map::emplace.
    ngg is 2 (3 for the 5th-order schemes, inviscid_scheme / 10 == 5)."""
    par = {}
    for name in SETUP_FILES:
        path = os.path.join(setup_dir, name)
        if not os.path.exists(path):
            continue
        for line in open(path):
            if line.startswith("//") or line.startswith("!") or not line.strip():
                continue
            toks = line.split()
            if len(toks) < 4:
                continue
            typ, key, val = toks[0], toks[1], toks[3]
            if key in par:
                continue
            if typ == "int":
                par[key] = int(val)
            elif typ == "double":
                par[key] = float(val)
            elif typ == "bool":
                par[key] = bool(int(val)) if val.isdigit() else val.lower() == "true"
            elif typ == "string":
                par[key] = val
    par.setdefault("ngg", 3 if par.get("inviscid_scheme", 0) // 10 == 5 else 2)
    return par


# ------------------------------------------------------------ mesh files

def _tokens(path):
    with open(path) as f:
        return f.read().split()


def read_grid(path):
    """[(dims, x, y, z)] with x, y, z as [mz][my][mx] arrays (Mesh.cpp:566-614)."""
    lines = open(path).read().splitlines()
    n_block = int(lines[0].split()[0])
    dims = [tuple(int(v) for v in lines[1 + b].split()[:3]) for b in range(n_block)]
    vals = np.array(" ".join(lines[1 + n_block:]).split(), dtype=np.float64)
    out, o = [], 0
    for mx, my, mz in dims:
        n = mx * my * mz
        xyz = [vals[o + q * n:o + (q + 1) * n].reshape(mz, my, mx) for q in range(3)]
        o += 3 * n
        out.append(((mx, my, mz), *xyz))
    return out


def read_boundary(path, n_block):
    """Per block the raw 7-integer boundary records (Mesh.cpp:616-636)."""
    lines = iter(open(path).read().splitlines())
    out = []
    for _ in range(n_block):
        n = int(next(lines).split()[0])
        out.append([[int(v) for v in next(lines).split()[:7]] for _ in range(n)])
    return out


def read_inner(path, n_block):
    """Per block the raw 13-integer interface records: six of the first line
    and seven of the second (Mesh.cpp:638-670)."""
    lines = open(path).read().splitlines()
    counts = [int(v) for v in lines[0].split()[:n_block]]
    it = iter(lines[2:])  # the count line and the line after it
    out = []
    for b in range(n_block):
        faces = []
        for _ in range(counts[b]):
            a = [int(v) for v in next(it).split()[:7]]
            t = [int(v) for v in next(it).split()[:7]]
            faces.append(a[:6] + t)
        out.append(faces)
    return out


def ghost_grid(blocks, inner_faces, ngg=2, reference_ghosts=False):
    """Coordinates with ngg+1 ghost layers per block (Mesh.cpp:718-923):
    reflection across each face, interface ghosts copied from the neighbour
    block, edges and corners by the parallelogram rule.  blocks: [(dims, x,
    y, z)]; inner_faces: per block the raw 13-integer records.  Returns per
    block (X, Y, Z) arrays [mz+2g][my+2g][mx+2g], g = ngg + 1.

    The reference copies the neighbour's coordinates as they are.  Across a
    periodic interface (a block joined to the far end of the domain, itself
    included) those lie one period away, so the ghost layer jumps by the
    period and the central-difference metrics of the layers next to it go
    wrong (the Jacobian changes sign).  By default the copied ghosts are
    translated by the offset between the two coincident face layers, which
    is zero for a conforming interface and the period for a periodic one;
    reference_ghosts=True keeps the raw copy."""
    import combustioncodegpu_b200 as cc

    g = ngg + 1
    dim3 = blocks[0][0][2] > 1
    out = []
    for (mx, my, mz), x, y, z in blocks:
        arrs = []
        for a in (x, y, z):
            A = np.zeros((mz + 2 * g, my + 2 * g, mx + 2 * g))
            A[g:g + mz, g:g + my, g:g + mx] = a
            arrs.append(A)
        out.append(arrs)

    def at(A, i, j, k):  # reference (i, j, k) indexing with ghosts
        return A[k + g, j + g, i + g]

    def put(A, i, j, k, v):
        A[k + g, j + g, i + g] = v

    for b, ((mx, my, mz), _, _, _) in enumerate(blocks):
        for q, A in enumerate(out[b]):
            for k in range(mz):
                for j in range(my):
                    for i in range(-1, -g - 1, -1):
                        put(A, i, j, k, 2 * at(A, 0, j, k) - at(A, -i, j, k))
                    for i in range(mx, mx + g):
                        put(A, i, j, k, 2 * at(A, mx - 1, j, k) - at(A, 2 * (mx - 1) - i, j, k))
            for k in range(mz):
                for i in range(mx):
                    for j in range(-1, -g - 1, -1):
                        put(A, i, j, k, 2 * at(A, i, 0, k) - at(A, i, -j, k))
                    for j in range(my, my + g):
                        put(A, i, j, k, 2 * at(A, i, my - 1, k) - at(A, i, 2 * (my - 1) - j, k))
            for j in range(my):
                for i in range(mx):
                    for k in range(-1, -g - 1, -1):
                        if dim3:
                            put(A, i, j, k, 2 * at(A, i, j, 0) - at(A, i, j, -k))
                        else:
                            put(A, i, j, k, at(A, i, j, 0) + (k if q == 2 else 0))
                    for k in range(mz, mz + g):
                        if dim3:
                            put(A, i, j, k, 2 * at(A, i, j, mz - 1) - at(A, i, j, 2 * (mz - 1) - k))
                        else:
                            put(A, i, j, k, at(A, i, j, mz - 1) + ((k - mz + 1) if q == 2 else 0))
    # interface ghosts from the neighbour (Mesh.cpp:874-923)
    for b, faces in enumerate(inner_faces):
        for raw in faces:
            fc = cc.register_inner_face(raw, ngg)
            nb = out[fc.target_block]
            mn = list(fc.range_start)
            mxr = list(fc.range_end)
            mt = list(fc.target_start)
            shift = -1 if fc.direction < 0 else 1
            mn[fc.face] += shift
            mxr[fc.face] += shift
            mt[fc.target_face] += -1 if fc.target_direction > 0 else 1
            ld, tld, st = list(fc.loop_dir), list(fc.target_loop_dir), list(fc.src_tar)
            # translation between the coincident face layers, measured at a
            # point of this block's face layer with interior tangential indices
            rs, re, ts = list(fc.range_start), list(fc.range_end), list(fc.target_start)
            pt = [min(max((rs[a] + re[a]) // 2, 0), blocks[b][0][a] - 1) for a in range(3)]
            pt[fc.face] = re[fc.face] if fc.direction < 0 else rs[fc.face]
            dd = [pt[a] - rs[a] for a in range(3)]
            tp = [ts[a] + tld[a] * dd[st[a]] for a in range(3)]
            off = [0.0 if reference_ghosts else at(out[b][q], *pt) - at(nb[q], *tp) for q in range(3)]
            i1 = mn[0]
            while ld[0] * (i1 - mxr[0]) != 1:
                j1 = mn[1]
                while ld[1] * (j1 - mxr[1]) != 1:
                    k1 = mn[2]
                    while ld[2] * (k1 - mxr[2]) != 1:
                        di = [i1 - mn[0], j1 - mn[1], k1 - mn[2]]
                        i2 = mt[0] + tld[0] * di[st[0]]
                        j2 = mt[1] + tld[1] * di[st[1]]
                        k2 = mt[2] + tld[2] * di[st[2]]
                        for q in range(3):
                            put(out[b][q], i1, j1, k1, at(nb[q], i2, j2, k2) + off[q])
                        k1 += ld[2]
                    j1 += ld[1]
                i1 += ld[0]
    # edges and corners (parallelogram rule)
    for b, ((mx, my, mz), _, _, _) in enumerate(blocks):
        for A in out[b]:
            for i in range(1, g + 1):
                for j in range(1, g + 1):
                    for k in range(mz):
                        i1, j1, i2, j2 = -i, -j, mx - 1 + i, my - 1 + j
                        put(A, i1, j1, k, at(A, i1, 0, k) + at(A, 0, j1, k) - at(A, 0, 0, k))
                        put(A, i2, j2, k, at(A, i2, my - 1, k) + at(A, mx - 1, j2, k) - at(A, mx - 1, my - 1, k))
                        put(A, i1, j2, k, at(A, i1, my - 1, k) + at(A, 0, j2, k) - at(A, 0, my - 1, k))
                        put(A, i2, j1, k, at(A, i2, 0, k) + at(A, mx - 1, j1, k) - at(A, mx - 1, 0, k))
            for i in range(1, g + 1):
                for j in range(my):
                    for k in range(1, g + 1):
                        i1, k1, i2, k2 = -i, -k, mx - 1 + i, mz - 1 + k
                        put(A, i1, j, k1, at(A, i1, j, 0) + at(A, 0, j, k1) - at(A, 0, j, 0))
                        put(A, i2, j, k2, at(A, i2, j, mz - 1) + at(A, mx - 1, j, k2) - at(A, mx - 1, j, mz - 1))
                        put(A, i1, j, k2, at(A, i1, j, mz - 1) + at(A, 0, j, k2) - at(A, 0, j, mz - 1))
                        put(A, i2, j, k1, at(A, i2, j, 0) + at(A, mx - 1, j, k1) - at(A, mx - 1, j, 0))
            for i in range(-g, mx + g):
                for j in range(1, g + 1):
                    for k in range(1, g + 1):
                        j1, k1, j2, k2 = -j, -k, my - 1 + j, mz - 1 + k
                        put(A, i, j1, k1, at(A, i, j1, 0) + at(A, i, 0, k1) - at(A, i, 0, 0))
                        put(A, i, j2, k2, at(A, i, j2, mz - 1) + at(A, i, my - 1, k2) - at(A, i, my - 1, mz - 1))
                        put(A, i, j1, k2, at(A, i, j1, mz - 1) + at(A, i, 0, k2) - at(A, i, 0, mz - 1))
                        put(A, i, j2, k1, at(A, i, j2, 0) + at(A, i, my - 1, k1) - at(A, i, my - 1, 0))
    return out


# ---------------------------------------------------- boundary conditions

def _sections(path):
    """{label: {name: value}} of a per-label file ("label n" opens a section,
    "double key = v", "option key = v", "species NAME = v" lines; "end")."""
    out, cur = {}, None
    if not os.path.exists(path):
        return out
    for line in open(path):
        toks = line.lower().split()
        if not toks or toks[0].startswith("//"):
            continue
        if toks[0] == "end":
            break
        if toks[0] == "label":
            cur = out.setdefault(int(toks[1]), {"double": {}, "option": {}, "species": {}})
            continue
        if cur is not None and toks[0] in ("double", "option", "species") and len(toks) >= 4:
            key = line.split()[1].upper() if toks[0] == "species" else toks[1]
            cur[toks[0]][key] = toks[3] if toks[0] == "option" else float(toks[3])
    return out


def read_conditions(setup_dir, labels, species=None):
    """Boundary conditions of the labels the boundary file uses
    (BoundCond.cu:315-409): type from 5_boundary_condition.txt, else by label
    (2 wall, 5 inflow, 6 outflow); wall values from 7_wall.txt
    (BoundCond.cpp:107-137), inflow values from 6_inflow.txt
    (BoundCond.cpp:10-104, the (mach | velocity, pressure, temperature |
    density) combinations)."""
    kinds = {}
    path = os.path.join(setup_dir, "5_boundary_condition.txt")
    if os.path.exists(path):
        for line in open(path):
            toks = line.lower().split()
            if not toks or toks[0].startswith("//"):
                continue
            if toks[0] == "end":
                break
            if toks[0] in BC_KIND and len(toks) >= 3 and int(toks[2]) in labels:
                kinds.setdefault(int(toks[2]), BC_KIND[toks[0]])
    for lab in labels:
        if lab not in kinds and lab in (2, 5, 6):
            kinds[lab] = lab
    walls = _sections(os.path.join(setup_dir, "7_wall.txt"))
    inflows = _sections(os.path.join(setup_dir, "6_inflow.txt"))
    bcs = []
    for lab in sorted(kinds):
        kind = kinds[lab]
        bc = {"label": lab, "kind": kind}
        if kind == 2:
            w = walls.get(lab, {"double": {}, "option": {}})
            iso = w["option"].get("thermal_type", "isothermal") == "isothermal"
            bc["thermal_type"] = 0 if iso else 1
            bc["t_wall"] = w["double"].get("temperature", 300.0)
        elif kind == 5:
            bc.update(inflow_state(inflows.get(lab, {"double": {}, "species": {}}), species))
        bcs.append(bc)
    return bcs


def inflow_state(sec, species):
    """Primitive state of an inflow section (BoundCond.cpp:10-104)."""
    d = sec["double"]
    mach, vel = d.get("mach", -1.0), d.get("velocity", -1.0)
    p, T, rho = d.get("pressure", 101325.0), d.get("temperature", -1.0), d.get("density", -1.0)
    if species is None:
        yk, mw, gamma = [], cases.MW_AIR, cases.GAMMA_AIR
    else:
        names = list(species["names"])
        yk = np.zeros(len(names))
        for nm, v in sec.get("species", {}).items():
            if nm in names:
                yk[names.index(nm)] = v
        mw = 1.0 / float(np.sum(yk / species["mw"]))
        gamma = None
    if T < 0:
        T = p * mw / (rho * cases.R_U)
    if gamma is None:
        cp = cv = 0.0
        for k in range(len(yk)):
            lo = species["low_temp_coeff"][k] if T < species["t_mid"][k] else species["high_temp_coeff"][k]
            te = max(T, species["t_low"][k])
            c = sum(lo[q] * te ** q for q in range(5)) * cases.R_U / species["mw"][k]
            cp += yk[k] * c
            cv += yk[k] * (c - cases.R_U / species["mw"][k])
        gamma = cp / cv
    c = float(np.sqrt(gamma * cases.R_U / mw * T))
    vel = mach * c if mach >= 0 else vel
    if rho < 0:
        rho = p * mw / (cases.R_U * T)
    return {"density": rho, "u": d.get("u", 1.0) * vel, "v": d.get("v", 0.0) * vel, "w": d.get("w", 0.0) * vel,
            "pressure": p, "temperature": T, "yk": list(yk)}


# -------------------------------------------------------------- whole case

def load_case(input_dir, ngg=None, reference_ghosts=False):
    """A reference input_files/ directory as a case dict for Driver.from_case.
    The initial state is the first group of 8_initialization.txt (a uniform
    inflow state over the domain, Initialize.cu:24-120; patches beyond the
    first group are not applied)."""
    setup = os.path.join(input_dir, "setup")
    par = read_parameters(setup)
    ngg = ngg or par["ngg"]
    species = None
    if par.get("n_spec", 0) > 0 or "mechanism_file" in par:
        rd = lambda key: open(os.path.join(input_dir, par[key])).read()
        species = cases.parse_chemdata(rd("mechanism_file"), rd("therm_file"), rd("transport_file"))
    grid = read_grid(os.path.join(input_dir, "grid", "grid%4d.grd" % 0))
    nb = len(grid)
    bnd = read_boundary(os.path.join(input_dir, "boundary_condition", "boundary%4d.txt" % 0), nb)
    inner_path = os.path.join(input_dir, "boundary_condition", "inner%4d.txt" % 0)
    inner = read_inner(inner_path, nb) if os.path.exists(inner_path) else [[] for _ in range(nb)]
    coords = ghost_grid(grid, inner, ngg, reference_ghosts)
    labels = sorted({r[6] for faces in bnd for r in faces})
    bcs = read_conditions(setup, labels, species)
    init = initial_state(setup, species)
    params = cases.default_params(species, viscous=par.get("viscous_order", 2) > 0, cfl=par.get("cfl", 0.5))
    for key in ("inviscid_scheme", "reconstruction", "limiter", "viscous_order", "prandtl_number",
                "schmidt_number"):
        if key in par:
            params[key] = par[key]
    params["ngg"] = ngg
    blocks = []
    for ((dims), _, _, _), (X, Y, Z), braw, iraw in zip(grid, coords, bnd, inner):
        jac, met = cases.jac_metric(X, Y, Z, ngg)
        ng = (dims[0] + 2 * ngg) * (dims[1] + 2 * ngg) * (dims[2] + 2 * ngg)
        bv = np.tile(np.array([init["density"], init["u"], init["v"], init["w"], init["pressure"],
                               init["temperature"]])[:, None], ng)
        yk = np.tile(np.asarray(init["yk"], dtype=np.float64)[:, None], ng)
        blocks.append({"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk, "boundaries": braw,
                       "inner_faces": iraw})
    return {"name": os.path.basename(os.path.normpath(input_dir)), "params": params, "blocks": blocks,
            "bcs": bcs, "parameters": par}


def initial_state(setup_dir, species):
    """The inflow state of the first initialization group (Initialize.cu:24-60)."""
    path = os.path.join(setup_dir, "8_initialization.txt")
    label = None
    if os.path.exists(path):
        for line in open(path):
            toks = line.lower().split()
            if len(toks) >= 2 and toks[0] == "label":
                label = int(toks[1])
                break
    inflows = _sections(os.path.join(setup_dir, "6_inflow.txt"))
    sec = inflows.get(label) if label is not None else None
    if sec is None and inflows:
        sec = inflows[sorted(inflows)[0]]
    if sec is None:
        raise ValueError("no initial state: 8_initialization.txt names no label of 6_inflow.txt")
    return inflow_state(sec, species)


def write_case(case, input_dir, coords, init_state=None):
    """Write a case dict in the reference's formats.  coords: per block the
    interior coordinates (x, y, z), each [mz][my][mx].  init_state (a dict
    with density, u, v, w, pressure, temperature, yk) becomes inflow label
    1000, which 8_initialization.txt names; boundary condition values go to
    6_inflow.txt / 7_wall.txt."""
    os.makedirs(os.path.join(input_dir, "grid"), exist_ok=True)
    os.makedirs(os.path.join(input_dir, "boundary_condition"), exist_ok=True)
    os.makedirs(os.path.join(input_dir, "setup"), exist_ok=True)
    blocks = case["blocks"]
    with open(os.path.join(input_dir, "grid", "grid%4d.grd" % 0), "w") as f:
        f.write("%d\n" % len(blocks))
        for b in blocks:
            f.write("%d %d %d\n" % tuple(b["dims"]))
        for xyz in coords:
            for a in xyz:
                f.write("\n".join("%.17g" % v for v in np.asarray(a).ravel()) + "\n")
    with open(os.path.join(input_dir, "boundary_condition", "boundary%4d.txt" % 0), "w") as f:
        for b in blocks:
            f.write("%d\n" % len(b["boundaries"]))
            for r in b["boundaries"]:
                f.write(" ".join(str(int(v)) for v in r) + "\n")
    with open(os.path.join(input_dir, "boundary_condition", "inner%4d.txt" % 0), "w") as f:
        f.write(" ".join(str(len(b["inner_faces"])) for b in blocks) + "\n\n")
        for b in blocks:
            for r in b["inner_faces"]:
                f.write(" ".join(str(int(v)) for v in r[:6]) + " -1\n")
                f.write(" ".join(str(int(v)) for v in r[6:13]) + "\n")
    p = case["params"]
    sp = p.get("species")
    with open(os.path.join(input_dir, "setup", "2_scheme.txt"), "w") as f:
        for key in ("inviscid_scheme", "reconstruction", "limiter", "viscous_order"):
            f.write("int %s = %d\n" % (key, p[key]))
        f.write("double cfl = %.17g\n" % p["cfl"])
    with open(os.path.join(input_dir, "setup", "9_transport_property.txt"), "w") as f:
        f.write("double prandtl_number = %.17g\ndouble schmidt_number = %.17g\n" % (p["prandtl_number"],
                                                                              p["schmidt_number"]))
    with open(os.path.join(input_dir, "setup", "3_species_reactions.txt"), "w") as f:
        f.write("int n_spec = %d\n" % (0 if sp is None else sp["n_spec"]))
        if sp is not None:
            f.write("string mechanism_file = chemistry/mech.inp\nstring therm_file = chemistry/therm.dat\n"
                    "string transport_file = chemistry/tran.dat\n")
    if sp is not None:
        os.makedirs(os.path.join(input_dir, "chemistry"), exist_ok=True)
        for key, fn in (("mechanism", "mech.inp"), ("therm", "therm.dat"), ("tran", "tran.dat")):
            open(os.path.join(input_dir, "chemistry", fn), "w").write(sp["texts"][key])
    names = [] if sp is None else list(sp["names"])

    def inflow_lines(lab, st):
        out = ["label %d" % lab, "double density = %.17g" % st["density"], "double velocity = 1.0",
               "double u = %.17g" % st["u"], "double v = %.17g" % st["v"], "double w = %.17g" % st["w"],
               "double pressure = %.17g" % st["pressure"], "double temperature = %.17g" % st["temperature"]]
        out += ["species %s = %.17g" % (n, y) for n, y in zip(names, st.get("yk", []))]
        return out

    inflow, wall, bcl = [], [], []
    for bc in case["bcs"]:
        kind = {2: "wall", 5: "inflow", 6: "outflow"}[bc["kind"]]
        bcl.append("%s %s_%d %d" % (kind, kind, bc["label"], bc["label"]))
        if bc["kind"] == 2:
            wall += ["label %d" % bc["label"], "option thermal_type = %s" % (
                "isothermal" if bc.get("thermal_type", 0) == 0 else "adiabatic"),
                "double temperature = %.17g" % bc.get("t_wall", 300.0)]
        elif bc["kind"] == 5:
            inflow += inflow_lines(bc["label"], bc)
    if init_state is not None:
        inflow = inflow_lines(1000, init_state) + inflow
    open(os.path.join(input_dir, "setup", "5_boundary_condition.txt"), "w").write("\n".join(bcl + ["end"]) + "\n")
    open(os.path.join(input_dir, "setup", "6_inflow.txt"), "w").write("\n".join(inflow + ["end"]) + "\n")
    open(os.path.join(input_dir, "setup", "7_wall.txt"), "w").write("\n".join(wall + ["end"]) + "\n")
    open(os.path.join(input_dir, "setup", "8_initialization.txt"), "w").write(
        "int n_group = 1\nlabel 1000\nend\n")
