"""Inputs of the residual path: species data, grids, face descriptors, fields.

Species data.  The 9-species H2/O2/N2 data files the workloads name (NASA-7
thermo and Lennard-Jones transport in the reference's ChemData format) are
not available offline, so `synthetic_species()` builds a clearly labelled
SYNTHETIC set:
  * molecular weights from the reference's own element table
    (Element.cpp:13-132: H 1.008, N 14.007, O 15.999), summed in the
    reference's element-map order (ChemData.cpp:160-166);
  * cp/R from a rigid-rotor + Einstein-oscillator model with seeded mode
    temperatures, least-squares fitted by NASA-7 polynomials on
    [200, 1000] K and [1000, 3500] K, enthalpy offsets chosen for continuity
    at 1000 K and seeded formation enthalpies;
  * seeded Lennard-Jones well depths and diameters;
  * every coefficient is written in the CHEMKIN text layout that
    ChemData.cpp:106-228 reads (E15.8 fields) and read back, so the arrays
    are exactly what the reference would load from these files.
Physical realism is not claimed; the CUDA path and the oracle read the same
numbers, so parity does not depend on it.

Grids.  The reference is vertex-centred (Mesh.cpp:226-488): a block of m
points along an axis of length L has spacing L/(m-1), and a periodic axis is
an interface of the block with itself that shares the end layer
(Mesh.cpp:35-143, Field.cu:213-266).  Metrics and Jacobian follow the
reference's central-difference formulas, ghost points included.
"""
import math

import numpy as np

R_U = 8314.462618       # Constants.h:19
GAMMA_AIR = 1.4         # Constants.h:23
MW_AIR = 28.9647        # Constants.h:28
ATOMIC_WEIGHT = {"H": 1.008, "N": 14.007, "O": 15.999}  # Element.cpp:14-21

H2O2_N2_SPECIES = [
    ("H2", {"H": 2}), ("O2", {"O": 2}), ("H2O", {"H": 2, "O": 1}), ("OH", {"O": 1, "H": 1}),
    ("H", {"H": 1}), ("O", {"O": 1}), ("HO2", {"H": 1, "O": 2}), ("H2O2", {"H": 2, "O": 2}),
    ("N2", {"N": 2}),
]

T_LOW, T_MID, T_HIGH = 200.0, 1000.0, 3500.0


def _cp_model(n_atoms, linear, thetas, T):
    """cp/R of a rigid rotor plus Einstein oscillators."""
    if n_atoms == 1:
        return np.full_like(T, 2.5)
    base = 3.5 if linear else 4.0
    x = thetas[:, None] / T[None, :]
    ex = np.exp(np.minimum(x, 700.0))
    return base + np.sum(x * x * ex / (ex - 1.0) ** 2, axis=0)


def _fmt_e15(v):
    s = "%15.8E" % v
    assert len(s) == 15
    return s


def synthetic_species(species=H2O2_N2_SPECIES, seed=2024):
    """Synthetic species tables (see module docstring).  Returns a dict with the
    DParameter arrays and the ChemData-format file texts."""
    rng = np.random.default_rng(seed)
    ns = len(species)
    names = [s[0] for s in species]
    elements = sorted({e for _, comp in species for e in comp})  # std::map order
    mw = np.zeros(ns)
    for k, (_, comp) in enumerate(species):
        w = 0.0
        for e in elements:
            w += ATOMIC_WEIGHT[e] * comp.get(e, 0)
        mw[k] = w
    Tlo = np.linspace(T_LOW, T_MID, 161)
    Thi = np.linspace(T_MID, T_HIGH, 201)
    low = np.zeros((ns, 7))
    high = np.zeros((ns, 7))
    for k, (name, comp) in enumerate(species):
        n_atoms = sum(comp.values())
        linear = n_atoms <= 2
        n_modes = 0 if n_atoms == 1 else (3 * n_atoms - 5 if linear else 3 * n_atoms - 6)
        thetas = rng.uniform(900.0, 6000.0, size=max(n_modes, 1))[:n_modes]
        hf_R = 0.0 if name in ("H2", "O2", "N2") else float(rng.uniform(-3.0e4, 3.0e4))
        for T, out in ((Tlo, low), (Thi, high)):
            A = np.vstack([T ** p for p in range(5)]).T
            cp = _cp_model(n_atoms, linear, thetas, T)
            out[k, :5] = np.linalg.lstsq(A, cp, rcond=None)[0]
        # cp continuous at T_mid: shift the high-range constant term
        at_mid = lambda c: sum(c[p] * T_MID ** p for p in range(5))
        high[k, 0] += at_mid(low[k]) - at_mid(high[k])

        def h_poly(c, T):
            return c[0] * T + c[1] * T ** 2 / 2 + c[2] * T ** 3 / 3 + c[3] * T ** 4 / 4 + c[4] * T ** 5 / 5

        low[k, 5] = hf_R - h_poly(low[k], 298.15)
        high[k, 5] = h_poly(low[k], T_MID) + low[k, 5] - h_poly(high[k], T_MID)
        low[k, 6] = 0.0
        high[k, 6] = 0.0
    eps_k = rng.uniform(30.0, 600.0, size=ns)
    sigma = rng.uniform(2.0, 4.0, size=ns)

    # CHEMKIN texts (ChemData.cpp:10-61 mechanism, 106-228 therm, 230-261 tran)
    mech = ["ELEMENTS", "--------", "%d" % len(elements), "--------", " ".join(elements), "SPECIES",
            "------------------", "%d" % ns, "------------------", " ".join(names), "REACTIONS", "END"]
    therm = ["THERMO", "%10.3f%10.3f%10.3f" % (T_LOW, T_MID, T_HIGH)]
    for k, (name, comp) in enumerate(species):
        head = name.ljust(18) + " " * 6
        ce = ""
        for e in elements:
            if comp.get(e, 0):
                ce += ("%-2s%3d" % (e, comp[e]))
        ce = ce.ljust(20)[:20]
        head = (head + ce + "G").ljust(45)
        head += "%10.3f%10.3f%8.2f" % (T_LOW, T_HIGH, T_MID)
        head = head.ljust(79) + "1"
        therm.append(head)
        c = list(high[k, :5])
        therm.append("".join(_fmt_e15(v) for v in c) + "    2")
        c = [high[k, 5], high[k, 6], low[k, 0], low[k, 1], low[k, 2]]
        therm.append("".join(_fmt_e15(v) for v in c) + "    3")
        c = [low[k, 3], low[k, 4], low[k, 5], low[k, 6]]
        therm.append("".join(_fmt_e15(v) for v in c) + "                   4")
    therm.append("END")
    tran = ["%-16s%4d%10.3f%10.3f%10.3f%10.3f%10.3f" % (n, 1, e, s, 0.0, 0.0, 0.0)
            for n, e, s in zip(names, eps_k, sigma)]
    tran.append("END")
    texts = {"mechanism": "\n".join(mech) + "\n", "therm": "\n".join(therm) + "\n", "tran": "\n".join(tran) + "\n"}
    return parse_chemdata(texts["mechanism"], texts["therm"], texts["tran"], texts)


def parse_chemdata(mech_text, therm_text, tran_text, texts=None):
    """Species arrays from ChemData-format texts (restates ChemData.cpp:10-261:
    mechanism species order, fixed-column NASA-7 records, LJ parameters and the
    derived Wilke constants)."""
    lines = mech_text.splitlines()
    n_elem = int(lines[2].split()[0])
    i = 4
    elements = []
    while lines[i].split()[0].upper() != "SPECIES":
        elements += lines[i].upper().split()
        i += 1
    elem_list = sorted(set(elements))
    i += 2
    ns = int(lines[i].split()[0])
    i += 2
    names = []
    while True:
        toks = lines[i].upper().split()
        if toks and toks[0] == "REACTIONS":
            break
        names += toks
        i += 1
    names = names[:ns]
    index = {n: k for k, n in enumerate(names)}
    tl = therm_text.splitlines()
    j = 0
    while not tl[j].upper().startswith("THERMO"):
        j += 1
    glob = [float(v) for v in tl[j + 1].split()[:3]]
    t_low = np.full(ns, glob[0])
    t_mid = np.full(ns, glob[1])
    t_high = np.full(ns, glob[2])
    low = np.zeros((ns, 7))
    high = np.zeros((ns, 7))
    mw = np.zeros(ns)
    j += 2
    while j < len(tl) and not tl[j].upper().startswith("END"):
        line = tl[j]
        if not line.strip() or line.startswith("!"):
            j += 1
            continue
        name = line[:18].split()[0].upper()
        if name not in index:
            j += 4
            continue
        k = index[name]
        t_low[k] = float(line[45:55])
        t_high[k] = float(line[55:65])
        mid = line[65:75].strip()
        if mid:
            t_mid[k] = float(mid.split()[0])
        comp = {}
        for q in range(4):
            s = line[24 + 5 * q:29 + 5 * q].strip()
            if not s or s.startswith("0"):
                break
            toks = s.split()
            comp[toks[0].upper()] = int(toks[1])
        w = 0.0
        for e in elem_list:
            w += ATOMIC_WEIGHT[e] * comp.get(e, 0)
        mw[k] = w
        l2, l3, l4 = tl[j + 1], tl[j + 2], tl[j + 3]
        f = lambda s, q: float(s[15 * q:15 * q + 15])
        high[k, :5] = [f(l2, q) for q in range(5)]
        high[k, 5], high[k, 6], low[k, 0], low[k, 1], low[k, 2] = [f(l3, q) for q in range(5)]
        low[k, 3], low[k, 4], low[k, 5], low[k, 6] = [f(l4, q) for q in range(4)]
        j += 4
    LJ_inv = np.zeros(ns)
    vis_coeff = np.zeros(ns)
    for line in tran_text.splitlines():
        toks = line.upper().split()
        if not toks or toks[0].startswith("END"):
            continue
        if toks[0] in index:
            k = index[toks[0]]
            eps, sig = float(toks[2]), float(toks[3])
            LJ_inv[k] = 1.0 / eps
            vis_coeff[k] = 2.6693e-6 * math.sqrt(mw[k]) / (sig * sig)
    Wj = np.zeros((ns, ns))
    Sw = np.zeros((ns, ns))
    for a in range(ns):
        for b in range(ns):
            Wj[a, b] = (mw[b] / mw[a]) ** 0.25
            Sw[a, b] = 1.0 / math.sqrt(8 * (1 + mw[a] / mw[b]))
    return {
        "names": names, "n_spec": ns, "mw": mw, "t_low": t_low, "t_mid": t_mid, "t_high": t_high,
        "low_temp_coeff": low, "high_temp_coeff": high, "LJ_potent_inv": LJ_inv, "vis_coeff": vis_coeff,
        "WjDivWi_to_One4th": Wj, "sqrt_WiDivWjPl1Mul8": Sw, "texts": texts,
        "synthetic": texts is not None,
    }


# ------------------------------------------------------------------- grids

def block_coordinates(m, lengths, ngg=2):
    """Uniform vertex-centred coordinates on the box with ngg+1 ghost layers,
    spacing L/(m-1) (the lattice continues into the ghosts, which is what
    Mesh::init_ghost_grid gives on a uniform grid)."""
    g = ngg + 1
    axes = []
    for n, L in zip(m, lengths):
        h = L / (n - 1)
        axes.append(np.arange(-g, n + g, dtype=np.float64) * h)
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return x, y, z


def jac_metric(x, y, z, ngg=2):
    """Jacobian and metrics by the central differences of Mesh.cpp:226-488
    on the ghosted box (input coordinates carry one extra layer).  Returns
    jac [Ng] and metric [9][Ng] in (k,j,i) C order = i fastest."""
    def d(a, axis):
        return (np.roll(a, -1, axis) - np.roll(a, 1, axis)) * 0.5
    dxd1, dyd1, dzd1 = d(x, 2), d(y, 2), d(z, 2)
    dxd2, dyd2, dzd2 = d(x, 1), d(y, 1), d(z, 1)
    dxd3, dyd3, dzd3 = d(x, 0), d(y, 0), d(z, 0)
    jac = (dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2
           - dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1)
    m = [
        (dyd2 * dzd3 - dyd3 * dzd2) / jac, (dxd3 * dzd2 - dxd2 * dzd3) / jac, (dxd2 * dyd3 - dxd3 * dyd2) / jac,
        (dyd3 * dzd1 - dyd1 * dzd3) / jac, (dxd1 * dzd3 - dxd3 * dzd1) / jac, (dxd3 * dyd1 - dxd1 * dyd3) / jac,
        (dyd1 * dzd2 - dyd2 * dzd1) / jac, (dxd2 * dzd1 - dxd1 * dzd2) / jac, (dxd1 * dyd2 - dxd2 * dyd1) / jac,
    ]
    sl = (slice(1, -1),) * 3
    jac = np.ascontiguousarray(jac[sl]).ravel()
    met = np.stack([np.ascontiguousarray(a[sl]).ravel() for a in m])
    return jac, met


FACE_AXES = {"i": 0, "j": 1, "k": 2}


def boundary_raw(dims, face, label):
    """Raw boundary record (x1,x2,y1,y2,z1,z2,type) of Mesh::read_boundary for
    face 'i-','i+','j-',... of a block with dims (mx,my,mz); 0-based."""
    ax = FACE_AXES[face[0]]
    lo = face[1] == "-"
    r = []
    for a in range(3):
        if a == ax:
            v = 0 if lo else dims[a] - 1
            r += [v, v]
        else:
            r += [0, dims[a] - 1]
    return r + [label]


def inner_face_raw(dims, face, target_dims, target_face, target_block):
    """Raw inner-face record of Mesh::read_inner_interface (13 ints, 1-based,
    the first tangential axis given negative) for face `face` of a block
    joined to `target_face` of block `target_block` (0-based), axes aligned."""
    def rec(d, f):
        ax = FACE_AXES[f[0]]
        tang = [a for a in range(3) if a != ax]
        r = [0] * 6
        v = 1 if f[1] == "-" else d[ax]
        r[2 * ax], r[2 * ax + 1] = v, v
        r[2 * tang[0]], r[2 * tang[0] + 1] = -1, -d[tang[0]]
        r[2 * tang[1]], r[2 * tang[1] + 1] = 1, d[tang[1]]
        return r
    return rec(dims, face) + rec(target_dims, target_face) + [target_block + 1]


def periodic_raw(dims, axis, block=0):
    """Both inner faces that make `axis` of a block periodic (shared end layer)."""
    a = "ijk"[axis]
    return [inner_face_raw(dims, a + "-", dims, a + "+", block), inner_face_raw(dims, a + "+", dims, a + "-", block)]


# ------------------------------------------------------------------ fields

def _box_index(dims, ngg):
    return [np.arange(-ngg, n + ngg) for n in dims]


def _wrap(idx, n, periodic):
    return np.mod(idx, n - 1) if periodic else idx


def fourier_field(rng, dims, periodic, ngg=2, kmax=4, n_modes=12):
    """Seeded sum of Fourier modes with integer wave vectors |k| <= kmax,
    normalised to [-1, 1], on the ghosted box.  Periodic axes are sampled at
    the wrapped index so images and the shared layer hold identical values."""
    idx = _box_index(dims, ngg)
    ph = []
    for a in range(3):
        n = dims[a]
        w = _wrap(idx[a], n, periodic[a]).astype(np.float64)
        ph.append(2 * math.pi * w / (n - 1))
    Z, Y, X = np.meshgrid(ph[2], ph[1], ph[0], indexing="ij")
    f = np.zeros_like(X)
    count = 0
    while count < n_modes:
        k = rng.integers(-kmax, kmax + 1, size=3)
        if not k.any() or np.linalg.norm(k) > kmax:
            continue
        amp = rng.uniform(0.2, 1.0)
        phase = rng.uniform(0, 2 * math.pi)
        f += amp * np.cos(k[0] * X + k[1] * Y + k[2] * Z + phase)
        count += 1
    f = f - f.min()
    f = 2 * f / max(f.max(), 1e-300) - 1
    return f.ravel()


def multispecies_fields(dims, species, seed=1234, periodic=(True, True, True), ngg=2,
                        t_range=(300.0, 1500.0), vel_amp=10.0):
    """Frozen-chemistry box fields: T in t_range, p = 101325 (1 +/- 0.05),
    positive renormalised Y_k from Fourier modes, Taylor-Green velocity.
    Returns bv [6][Ng], yk [ns][Ng]."""
    rng = np.random.default_rng(seed)
    ns = species["n_spec"]
    T = t_range[0] + (t_range[1] - t_range[0]) * 0.5 * (fourier_field(rng, dims, periodic, ngg) + 1)
    p = 101325.0 * (1 + 0.05 * fourier_field(rng, dims, periodic, ngg))
    Y = np.empty((ns, T.size))
    for k in range(ns):
        s = 2.0 * fourier_field(rng, dims, periodic, ngg)
        Y[k] = np.log1p(np.exp(s)) + 1e-3
    Y /= Y.sum(axis=0, keepdims=True)
    idx = _box_index(dims, ngg)
    ph = []
    for a in range(3):
        n = dims[a]
        ph.append(2 * math.pi * _wrap(idx[a], n, periodic[a]).astype(np.float64) / (n - 1))
    Z, Y3, X = np.meshgrid(ph[2], ph[1], ph[0], indexing="ij")
    u = (vel_amp * np.sin(X) * np.cos(Y3) * np.cos(Z)).ravel()
    v = (-vel_amp * np.cos(X) * np.sin(Y3) * np.cos(Z)).ravel()
    w = np.zeros_like(u)
    mw_inv = (Y / species["mw"][:, None]).sum(axis=0)
    rho = p / (R_U * T * mw_inv)
    return np.stack([rho, u, v, w, p, T]), Y


def sod_fields(dims, lengths, ngg=2):
    """Sod shock tube (air): rho=1, p=1e5 for x < L/2, rho=0.125, p=1e4
    beyond; u=v=w=0; T = p W_air/(rho R_u)."""
    x, _, _ = block_coordinates(dims, lengths, ngg)
    x = x[1:-1, 1:-1, 1:-1].ravel()
    left = x < 0.5 * lengths[0]
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0e5, 1.0e4)
    z = np.zeros_like(rho)
    T = p * MW_AIR / (rho * R_U)
    return np.stack([rho, z, z, z, p, T]), np.zeros((0, rho.size))


def make_block(dims, lengths, ngg=2):
    x, y, z = block_coordinates(dims, lengths, ngg)
    return jac_metric(x, y, z, ngg)


def default_params(species=None, viscous=True, cfl=0.5):
    """Scheme parameters with the reference's key names (2_scheme, 9_transport
    setup files): AUSM+ (3), MUSCL (2), minmod (0)."""
    return {
        "inviscid_scheme": 3, "reconstruction": 2, "limiter": 0,
        "viscous_order": 2 if viscous else 0, "cfl": cfl, "prandtl_number": 0.72,
        "schmidt_number": 0.9, "ngg": 2, "species": species,
    }


# --------------------------------------------------------------- workloads

def case_sod(mx=256, my=8, mz=8, lengths=(1.0, 0.03125, 0.03125)):
    """Sod shock tube on one block: outflow at both x ends, periodic y and z,
    air, inviscid, MUSCL-minmod, AUSM+, CFL 0.5."""
    dims = (mx, my, mz)
    jac, met = make_block(dims, lengths)
    bv, yk = sod_fields(dims, lengths)
    blk = {"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk,
           "boundaries": [boundary_raw(dims, "i-", 6), boundary_raw(dims, "i+", 6)],
           "inner_faces": periodic_raw(dims, 1) + periodic_raw(dims, 2)}
    return {"name": "sod", "params": default_params(None, viscous=False), "blocks": [blk],
            "bcs": [{"label": 6, "kind": 6}]}


def case_box(n=128, L=2e-3, species=None, seed=1234, viscous=True):
    """Periodic viscous frozen-chemistry box of n^3 points on an L cube."""
    species = species or synthetic_species()
    dims = (n, n, n)
    jac, met = make_block(dims, (L, L, L))
    bv, yk = multispecies_fields(dims, species, seed=seed)
    faces = []
    for a in range(3):
        faces += periodic_raw(dims, a)
    blk = {"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk, "boundaries": [], "inner_faces": faces}
    return {"name": "box%d" % n, "params": default_params(species, viscous=viscous), "blocks": [blk], "bcs": []}


def case_box_distorted(n=16, L=2e-3, amp=0.08, species=None, seed=21):
    """Periodic viscous box on a curvilinear grid: every coordinate is moved
    by a periodic sinusoid of the others (amplitude amp of a cell), so the
    metrics vary from point to point while the periodic continuation of the
    lattice into the ghosts stays exact."""
    species = species or synthetic_species()
    dims = (n, n, n)
    x, y, z = block_coordinates(dims, (L, L, L))
    h = L / (n - 1)
    w = 2 * math.pi / (h * (n - 1))  # one period across the block (the shared end layers coincide)
    xd = x + amp * h * np.sin(w * y) * np.cos(w * z)
    yd = y + amp * h * np.sin(w * z) * np.cos(w * x)
    zd = z + amp * h * np.sin(w * x) * np.cos(w * y)
    jac, met = jac_metric(xd, yd, zd)
    bv, yk = multispecies_fields(dims, species, seed=seed)
    faces = []
    for a in range(3):
        faces += periodic_raw(dims, a)
    blk = {"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk, "boundaries": [], "inner_faces": faces}
    return {"name": "box_distorted%d" % n, "params": default_params(species), "blocks": [blk], "bcs": []}


def case_multiblock(sizes_per_axis, L_cell=2e-3 / 127, species=None, seed=7):
    """Conforming periodic layout of blocks (a,b,c) = (nx_a, ny_b, nz_c);
    neighbouring blocks share their interface layer; the layout wraps
    periodically.  All blocks carry pieces of one global field."""
    species = species or synthetic_species()
    nxs, nys, nzs = sizes_per_axis
    na, nb, nc = len(nxs), len(nys), len(nzs)
    gdims = (sum(n - 1 for n in nxs) + 1, sum(n - 1 for n in nys) + 1, sum(n - 1 for n in nzs) + 1)
    gbv, gyk = multispecies_fields(gdims, species, seed=seed, ngg=2)
    G = [d + 4 for d in gdims]
    gbv = gbv.reshape(6, G[2], G[1], G[0])
    gyk = gyk.reshape(species["n_spec"], G[2], G[1], G[0])
    starts = [np.concatenate([[0], np.cumsum([n - 1 for n in s])[:-1]]) for s in (nxs, nys, nzs)]
    blocks = []
    bid = lambda a, b, c: a + na * (b + nb * c)
    for c in range(nc):
        for b in range(nb):
            for a in range(na):
                dims = (nxs[a], nys[b], nzs[c])
                jac, met = make_block(dims, tuple(L_cell * (d - 1) for d in dims))
                o = (starts[0][a], starts[1][b], starts[2][c])
                sl = (slice(None), slice(o[2], o[2] + dims[2] + 4), slice(o[1], o[1] + dims[1] + 4),
                      slice(o[0], o[0] + dims[0] + 4))
                bv = np.ascontiguousarray(gbv[sl]).reshape(6, -1)
                yk = np.ascontiguousarray(gyk[sl]).reshape(species["n_spec"], -1)
                faces = []
                nbr = [((a - 1) % na, b, c), ((a + 1) % na, b, c), (a, (b - 1) % nb, c), (a, (b + 1) % nb, c),
                       (a, b, (c - 1) % nc), (a, b, (c + 1) % nc)]
                for f, (nm, t) in enumerate(zip(["i-", "i+", "j-", "j+", "k-", "k+"], nbr)):
                    tdims = (nxs[t[0]], nys[t[1]], nzs[t[2]])
                    tf = nm[0] + ("+" if nm[1] == "-" else "-")
                    faces.append(inner_face_raw(dims, nm, tdims, tf, bid(*t)))
                blocks.append({"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk,
                               "boundaries": [], "inner_faces": faces})
    return {"name": "multiblock%d" % len(blocks), "params": default_params(species), "blocks": blocks,
            "bcs": [], "global_dims": gdims}


def multiblock_sizes(seed=2024, n_per_axis=4, lo=16, hi=96):
    """Block sizes of the uneven multiblock workload: n_per_axis sizes per
    axis drawn from U[lo, hi] (PCG64, seed); block (a, b, c) of the periodic
    layout is (nx_a, ny_b, nz_c), so every interface is conforming."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return tuple([int(v) for v in rng.integers(lo, hi + 1, size=n_per_axis)] for _ in range(3))


def case_multiblock64(seed=2024, species=None):
    """64 blocks (4 x 4 x 4 periodic layout) of 16..96 points per side."""
    return case_multiblock(multiblock_sizes(seed), species=species, seed=seed)


def mole_to_mass(X, mw):
    """Mass fractions of mole fractions X (any shape [ns, ...])."""
    X = np.asarray(X, dtype=np.float64)
    w = X * mw.reshape((-1,) + (1,) * (X.ndim - 1))
    return w / w.sum(axis=0, keepdims=True)


def case_mixing_layer(nx=1024, ny=512, nz=4, h=4e-3 / 1023, delta=1e-4, seed=11, species=None):
    """Temporal H2/air mixing layer (the precision-study workload).

    Fuel stream above the mid-plane: X(H2) = 0.3, X(N2) = 0.7, 300 K, u = 50
    m/s; oxidiser below: air as X(O2) = 0.21, X(N2) = 0.79, 600 K, u = 10 m/s;
    p = 101325 Pa.  The streams are blended with s = (1 + tanh((y - y_mid) /
    delta)) / 2 (u, T and the mass fractions linearly in s) and u, v carry
    seeded uniform perturbations of 1% of the velocity difference.  Uniform
    spacing h in all directions; periodic in x and z, zero-gradient outflow
    at both y ends."""
    species = species or synthetic_species()
    names = list(species["names"])
    mw = np.asarray(species["mw"])
    ns = len(names)
    x_fuel, x_ox = np.zeros(ns), np.zeros(ns)
    x_fuel[names.index("H2")], x_fuel[names.index("N2")] = 0.3, 0.7
    x_ox[names.index("O2")], x_ox[names.index("N2")] = 0.21, 0.79
    y_fuel, y_ox = mole_to_mass(x_fuel, mw), mole_to_mass(x_ox, mw)
    dims = (nx, ny, nz)
    lengths = (h * (nx - 1), h * (ny - 1), h * (nz - 1))
    jac, met = make_block(dims, lengths)
    _, yc, _ = block_coordinates(dims, lengths)
    yv = yc[1:-1, 1:-1, 1:-1].ravel()  # y of every ghosted point (i fastest)
    sfr = 0.5 * (1.0 + np.tanh((yv - 0.5 * lengths[1]) / delta))
    rng = np.random.Generator(np.random.PCG64(seed))
    du = 50.0 - 10.0
    u = 10.0 + du * sfr + 0.01 * du * rng.uniform(-1.0, 1.0, yv.size)
    v = 0.01 * du * rng.uniform(-1.0, 1.0, yv.size)
    w = np.zeros_like(u)
    T = 600.0 - 300.0 * sfr
    Y = y_ox[:, None] * (1.0 - sfr)[None, :] + y_fuel[:, None] * sfr[None, :]
    p = np.full_like(u, 101325.0)
    rho = p / (R_U * T * (Y / mw[:, None]).sum(axis=0))
    blk = {"dims": dims, "jac": jac, "metric": met, "bv": np.stack([rho, u, v, w, p, T]), "yk": Y,
           "boundaries": [boundary_raw(dims, "j-", 6), boundary_raw(dims, "j+", 6)],
           "inner_faces": periodic_raw(dims, 0) + periodic_raw(dims, 2)}
    return {"name": "mixing_layer%dx%dx%d" % dims, "params": default_params(species), "blocks": [blk],
            "bcs": [{"label": 6, "kind": 6}],
            "streams": {"fuel": {"X": x_fuel.tolist(), "T": 300.0, "u": 50.0},
                        "oxidiser": {"X": x_ox.tolist(), "T": 600.0, "u": 10.0}, "delta": delta}}


def case_channel(dims=(12, 9, 6), L=(2e-3, 1.5e-3, 1e-3), species=None, seed=99):
    """Inflow at i-, outflow at i+, isothermal wall at j-, adiabatic wall at
    j+, periodic k: exercises every boundary condition of the reference."""
    species = species or synthetic_species()
    jac, met = make_block(dims, L)
    bv, yk = multispecies_fields(dims, species, seed=seed, periodic=(False, False, True))
    Yin = np.zeros(16)
    ns = species["n_spec"]
    Yin[:ns] = 1.0 / ns
    rho_in = 101325.0 / (R_U * 600.0 * (Yin[:ns] / species["mw"]).sum())
    bcs = [{"label": 5, "kind": 5, "density": rho_in, "u": 20.0, "v": 0.0, "w": 0.0, "pressure": 101325.0,
            "temperature": 600.0, "yk": Yin},
           {"label": 6, "kind": 6},
           {"label": 2, "kind": 2, "thermal_type": 0, "t_wall": 500.0},
           {"label": 3, "kind": 2, "thermal_type": 1, "t_wall": 300.0}]
    blk = {"dims": dims, "jac": jac, "metric": met, "bv": bv, "yk": yk,
           "boundaries": [boundary_raw(dims, "i-", 5), boundary_raw(dims, "i+", 6),
                          boundary_raw(dims, "j-", 2), boundary_raw(dims, "j+", 3)],
           "inner_faces": periodic_raw(dims, 2)}
    return {"name": "channel", "params": default_params(species), "blocks": [blk], "bcs": bcs}
