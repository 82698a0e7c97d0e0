"""ctypes driver of the CPU FP64 oracle (cc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
check its CUDA result, and by bench.py for the CPU baseline.  The product never uses it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libcc_oracle.so")
_dp = ctypes.POINTER(ctypes.c_double)


def build():
    """gcc -O2 -fopenmp: FP contraction off so the restatement rounds like the
    reference's separate multiply/add sequence on the host."""
    src = os.path.join(HERE, "cc_oracle.c")
    hdr = os.path.join(HERE, "cc_oracle.h")
    os.makedirs(BUILD, exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(src), os.path.getmtime(hdr)):
        return LIB
    cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-Wall", "-o", LIB, src,
           "-lm"]
    subprocess.run(cmd, check=True)
    return LIB


class OcParams(ctypes.Structure):
    _fields_ = [("n_spec", ctypes.c_int), ("reconstruction", ctypes.c_int), ("limiter", ctypes.c_int),
                ("viscous_order", ctypes.c_int), ("ngg", ctypes.c_int), ("Pr", ctypes.c_double),
                ("cfl", ctypes.c_double), ("Sc", ctypes.c_double), ("mw", _dp), ("t_low", _dp),
                ("t_mid", _dp), ("t_high", _dp), ("low_coeff", _dp), ("high_coeff", _dp),
                ("LJ_potent_inv", _dp), ("vis_coeff", _dp), ("WjDivWi_to_One4th", _dp),
                ("sqrt_WiDivWjPl1Mul8", _dp)]


class OcBoundary(ctypes.Structure):
    _fields_ = [("range_start", ctypes.c_int * 3), ("range_end", ctypes.c_int * 3), ("type_label", ctypes.c_int),
                ("face", ctypes.c_int), ("direction", ctypes.c_int)]


class OcInnerFace(ctypes.Structure):
    _fields_ = [("range_start", ctypes.c_int * 3), ("range_end", ctypes.c_int * 3), ("face", ctypes.c_int),
                ("direction", ctypes.c_int), ("target_start", ctypes.c_int * 3), ("target_end", ctypes.c_int * 3),
                ("target_block", ctypes.c_int), ("target_face", ctypes.c_int), ("target_direction", ctypes.c_int),
                ("src_tar", ctypes.c_int * 3), ("loop_dir", ctypes.c_int * 3), ("target_loop_dir", ctypes.c_int * 3)]


class OcBc(ctypes.Structure):
    _fields_ = [("label", ctypes.c_int), ("kind", ctypes.c_int), ("thermal_type", ctypes.c_int),
                ("t_wall", ctypes.c_double), ("density", ctypes.c_double), ("u", ctypes.c_double),
                ("v", ctypes.c_double), ("w", ctypes.c_double), ("pressure", ctypes.c_double),
                ("temperature", ctypes.c_double), ("yk", ctypes.c_double * 32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        L = _lib
        L.oc_create.restype = ctypes.c_void_p
        L.oc_create.argtypes = [ctypes.POINTER(OcParams), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oc_destroy.argtypes = [ctypes.c_void_p]
        L.oc_set_threads.argtypes = [ctypes.c_int]
        for name in ("oc_add_boundary_raw", "oc_add_inner_face_raw"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oc_get_boundary.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OcBoundary)]
        L.oc_get_inner_face.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(OcInnerFace)]
        L.oc_add_bc.argtypes = [ctypes.c_void_p, ctypes.POINTER(OcBc)]
        L.oc_set_geometry.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.oc_set_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.oc_init.argtypes = [ctypes.c_void_p]
        L.oc_steady_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oc_rk3_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oc_lusgs_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oc_compute_dq.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.oc_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]
        L.oc_get_props.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
        L.oc_get_dt_local.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.oc_last_dt.argtypes = [ctypes.c_void_p]
        L.oc_last_dt.restype = ctypes.c_double
        L.oc_residual.argtypes = [ctypes.c_void_p, _dp]
        L.oc_newton_failures.argtypes = [ctypes.c_void_p]
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


class Oracle:
    """One oracle solver for a case dict (combustioncodegpu_b200.cases)."""

    def __init__(self, case, threads=None):
        L = lib()
        if threads:
            L.oc_set_threads(int(threads))
        prm = case["params"]
        sp = prm.get("species")
        self.ns = 0 if sp is None else int(sp["n_spec"])
        self._keep = []
        p = OcParams()
        p.n_spec = self.ns
        p.reconstruction = prm["reconstruction"]
        p.limiter = prm["limiter"]
        p.viscous_order = prm["viscous_order"]
        p.ngg = prm["ngg"]
        p.Pr = prm["prandtl_number"]
        p.cfl = prm["cfl"]
        p.Sc = prm["schmidt_number"]
        if self.ns:
            for fld, key in (("mw", "mw"), ("t_low", "t_low"), ("t_mid", "t_mid"), ("t_high", "t_high"),
                             ("low_coeff", "low_temp_coeff"), ("high_coeff", "high_temp_coeff"),
                             ("LJ_potent_inv", "LJ_potent_inv"), ("vis_coeff", "vis_coeff"),
                             ("WjDivWi_to_One4th", "WjDivWi_to_One4th"),
                             ("sqrt_WiDivWjPl1Mul8", "sqrt_WiDivWjPl1Mul8")):
                a = np.ascontiguousarray(sp[key], dtype=np.float64).ravel()
                self._keep.append(a)
                setattr(p, fld, _p(a))
        self.blocks = case["blocks"]
        dims = np.array([d for b in self.blocks for d in b["dims"]], dtype=np.int32)
        self.s = L.oc_create(ctypes.byref(p), len(self.blocks), dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        if not self.s:
            raise RuntimeError("oc_create failed")
        for bi, b in enumerate(self.blocks):
            for raw in b["boundaries"]:
                arr = (ctypes.c_int * 7)(*raw)
                assert L.oc_add_boundary_raw(self.s, bi, arr) == 0
            for raw in b["inner_faces"]:
                arr = (ctypes.c_int * 13)(*raw)
                assert L.oc_add_inner_face_raw(self.s, bi, arr) == 0
            jac = np.ascontiguousarray(b["jac"], dtype=np.float64)
            met = np.ascontiguousarray(b["metric"], dtype=np.float64)
            assert L.oc_set_geometry(self.s, bi, _p(jac), _p(met)) == 0
            bv = np.ascontiguousarray(b["bv"], dtype=np.float64)
            yk = np.ascontiguousarray(b["yk"], dtype=np.float64) if self.ns else None
            assert L.oc_set_state(self.s, bi, _p(bv), _p(yk)) == 0
        for d in case["bcs"]:
            bc = OcBc()
            bc.label, bc.kind = int(d["label"]), int(d["kind"])
            bc.thermal_type = int(d.get("thermal_type", 0))
            bc.t_wall = float(d.get("t_wall", 300.0))
            for k in ("density", "u", "v", "w", "pressure", "temperature"):
                setattr(bc, k, float(d.get(k, 0.0)))
            if "yk" in d:
                for i, v in enumerate(np.asarray(d["yk"])[: self.ns]):
                    bc.yk[i] = float(v)
            assert L.oc_add_bc(self.s, ctypes.byref(bc)) == 0

    def ng(self, bi):
        mx, my, mz = self.blocks[bi]["dims"]
        return (mx + 4) * (my + 4) * (mz + 4)

    def init(self):
        lib().oc_init(self.s)

    def steady_step(self, n=1, renorm_y=False):
        for _ in range(n):
            lib().oc_steady_step(self.s, 1 if renorm_y else 0)

    def lusgs_step(self, n=1, renorm_y=False):
        for _ in range(n):
            lib().oc_lusgs_step(self.s, 1 if renorm_y else 0)

    def rk3_step(self, n=1, renorm_y=False):
        for _ in range(n):
            lib().oc_rk3_step(self.s, 1 if renorm_y else 0)

    def dq(self, bi):
        mx, my, mz = self.blocks[bi]["dims"]
        out = np.empty((5 + self.ns, mx * my * mz))
        lib().oc_compute_dq(self.s, bi, _p(out))
        return out

    def state(self, bi):
        ng = self.ng(bi)
        bv = np.empty((6, ng))
        yk = np.empty((self.ns, ng))
        cv = np.empty((5 + self.ns, ng))
        lib().oc_get_state(self.s, bi, _p(bv), _p(yk) if self.ns else None, _p(cv))
        return bv, yk, cv

    def props(self, bi):
        ng = self.ng(bi)
        mul, cond, gam, ac = np.empty(ng), np.empty(ng), np.empty(ng), np.empty(ng)
        rd = np.empty((self.ns, ng))
        lib().oc_get_props(self.s, bi, _p(mul), _p(cond), _p(rd) if self.ns else None, _p(gam), _p(ac))
        return mul, cond, rd

    def dt_local(self, bi):
        mx, my, mz = self.blocks[bi]["dims"]
        out = np.empty(mx * my * mz)
        lib().oc_get_dt_local(self.s, bi, _p(out))
        return out

    def boundaries(self, bi):
        out = []
        i = 0
        while True:
            b = OcBoundary()
            if lib().oc_get_boundary(self.s, bi, i, ctypes.byref(b)) != 0:
                return out
            out.append(b)
            i += 1

    def inner_faces(self, bi):
        out = []
        i = 0
        while True:
            f = OcInnerFace()
            if lib().oc_get_inner_face(self.s, bi, i, ctypes.byref(f)) != 0:
                return out
            out.append(f)
            i += 1

    def last_dt(self):
        return lib().oc_last_dt(self.s)

    def residual(self):
        out = np.zeros(4)
        lib().oc_residual(self.s, _p(out))
        return out

    def newton_failures(self):
        return lib().oc_newton_failures(self.s)

    def close(self):
        if self.s:
            lib().oc_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_params(species, reconstruction=2, viscous_order=2, Pr=0.72, cfl=0.5, Sc=0.9):
    """OcParams for the known-answer hooks; returns (struct, keepalive)."""
    p = OcParams()
    p.n_spec = 0 if species is None else int(species["n_spec"])
    p.reconstruction, p.limiter, p.viscous_order, p.ngg = reconstruction, 0, viscous_order, 2
    p.Pr, p.cfl, p.Sc = Pr, cfl, Sc
    keep = []
    if p.n_spec:
        for fld, key in (("mw", "mw"), ("t_low", "t_low"), ("t_mid", "t_mid"), ("t_high", "t_high"),
                         ("low_coeff", "low_temp_coeff"), ("high_coeff", "high_temp_coeff"),
                         ("LJ_potent_inv", "LJ_potent_inv"), ("vis_coeff", "vis_coeff"),
                         ("WjDivWi_to_One4th", "WjDivWi_to_One4th"), ("sqrt_WiDivWjPl1Mul8", "sqrt_WiDivWjPl1Mul8")):
            a = np.ascontiguousarray(species[key], dtype=np.float64).ravel()
            keep.append(a)
            setattr(p, fld, _p(a))
    return p, keep


def kat_minmod(a, b):
    L = lib()
    L.oc_kat_minmod.restype = ctypes.c_double
    L.oc_kat_minmod.argtypes = [ctypes.c_double, ctypes.c_double]
    return L.oc_kat_minmod(a, b)


def kat_face_inviscid(species, pv4, k, reconstruction=2):
    """AUSM+ face flux from 4 points of primitives (rho,u,v,w,p,Y...) and a
    face normal k (metric row times J, equal on both sides)."""
    p, keep = make_params(species, reconstruction)
    pv = np.ascontiguousarray(pv4, dtype=np.float64)
    m = np.ascontiguousarray(k, dtype=np.float64)
    fc = np.zeros(5 + p.n_spec)
    L = lib()
    L.oc_kat_face_inviscid.argtypes = [ctypes.POINTER(OcParams), _dp, _dp, ctypes.c_double, _dp, ctypes.c_double, _dp]
    L.oc_kat_face_inviscid(ctypes.byref(p), _p(pv), _p(m), 1.0, _p(m), 1.0, _p(fc))
    return fc


def kat_h_cp(species, T):
    p, keep = make_params(species)
    h, cp = np.zeros(p.n_spec), np.zeros(p.n_spec)
    L = lib()
    L.oc_kat_h_cp.argtypes = [ctypes.POINTER(OcParams), ctypes.c_double, _dp, _dp]
    L.oc_kat_h_cp(ctypes.byref(p), float(T), _p(h), _p(cp))
    return h, cp


def kat_transport(species, T, Y, Sc=0.9):
    p, keep = make_params(species, Sc=Sc)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    mu, lam = ctypes.c_double(), ctypes.c_double()
    rd = np.zeros(p.n_spec)
    L = lib()
    L.oc_kat_transport.argtypes = [ctypes.POINTER(OcParams), ctypes.c_double, _dp, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double), _dp]
    L.oc_kat_transport(ctypes.byref(p), float(T), _p(Y), ctypes.byref(mu), ctypes.byref(lam), _p(rd))
    return mu.value, lam.value, rd


def kat_temperature(species, q5, Y, t0):
    p, keep = make_params(species)
    q = np.ascontiguousarray(q5, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    L = lib()
    L.oc_kat_temperature.restype = ctypes.c_double
    L.oc_kat_temperature.argtypes = [ctypes.POINTER(OcParams), _dp, _dp, ctypes.c_double]
    return L.oc_kat_temperature(ctypes.byref(p), _p(q), _p(Y), float(t0))


def kat_lusgs_jac_vec(Q, p, gam, psi, k, dQ):
    Q = np.ascontiguousarray(Q, dtype=np.float64)
    dQ = np.ascontiguousarray(dQ, dtype=np.float64)
    psi = np.ascontiguousarray(psi if len(psi) else [0.0], dtype=np.float64)
    k = np.ascontiguousarray(k, dtype=np.float64)
    dF = np.zeros_like(Q)
    L = lib()
    L.oc_kat_lusgs_jac_vec.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp]
    L.oc_kat_lusgs_jac_vec(len(Q), _p(Q), float(p), float(gam), _p(psi), _p(k), _p(dQ), _p(dF))
    return dF


def apply_boundaries(oracle):
    L = lib()
    L.oc_apply_boundaries.argtypes = [ctypes.c_void_p]
    return L.oc_apply_boundaries(oracle.s)
