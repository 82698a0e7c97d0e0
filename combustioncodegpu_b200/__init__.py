"""B200 (sm_100a) residual path of CombustionCodeGPU behind the reference's
Driver / Field / DParameter call surface.

The compute path is the in-tree CUDA library libcc_b200.so (C ABI declared in
include/cc_b200.h).  This module is the Python mirror of the reference's
host interface, bound with ctypes:

  reference (C++)                          here
  cfd::Parameter (Parameter.h:12-67)       Parameter (dict with get_int/...)
  cfd::Mesh / cfd::Block (Mesh.h:109-232)  Mesh / Block
  cfd::ChemData::spec (ChemData.h:11-61)   species dict (cases.synthetic_species)
  cfd::Driver (Driver.h:17-48)             Driver
  cfd::Field (Field.h:67-82)               Driver.field[b] (Field)

There is no CPU fallback: without the library, or without a device at
initialize_computation(), calls raise.
"""
import ctypes
import os

import numpy as np

from . import cases  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
# CC_LIBRARY selects another build of the library (the bounds-checked
# libcc_b200_bounds.so in its tests)
LIB_PATH = os.environ.get("CC_LIBRARY") or os.path.join(_HERE, "libcc_b200.so")
MAX_SPECIES = 16

CC_FP64, CC_MIXED, CC_FP32 = 0, 1, 2
CC_RK3, CC_STEADY_EULER, CC_STEADY_LUSGS = 0, 1, 2
PRECISIONS = {"fp64": CC_FP64, "mixed": CC_MIXED, "fp32": CC_FP32}
VARIANTS = ("l1", "tma", "split", "split-tma", "split-tma-p", "dq-tma")  # stage-kernel variants, cc_tuning order
SCHEMES = {"rk3": CC_RK3, "steady": CC_STEADY_EULER, "lusgs": CC_STEADY_LUSGS}

_dp = ctypes.POINTER(ctypes.c_double)


class CCParams(ctypes.Structure):
    _fields_ = [
        ("n_spec", ctypes.c_int), ("inviscid_scheme", ctypes.c_int), ("reconstruction", ctypes.c_int),
        ("limiter", ctypes.c_int), ("viscous_order", ctypes.c_int), ("ngg", ctypes.c_int),
        ("prandtl_number", ctypes.c_double), ("cfl", ctypes.c_double), ("schmidt_number", ctypes.c_double),
        ("mw", _dp), ("t_low", _dp), ("t_mid", _dp), ("t_high", _dp), ("low_temp_coeff", _dp),
        ("high_temp_coeff", _dp), ("LJ_potent_inv", _dp), ("vis_coeff", _dp), ("WjDivWi_to_One4th", _dp),
        ("sqrt_WiDivWjPl1Mul8", _dp),
    ]


class CCBoundary(ctypes.Structure):
    _fields_ = [("range_start", ctypes.c_int * 3), ("range_end", ctypes.c_int * 3), ("type_label", ctypes.c_int),
                ("face", ctypes.c_int), ("direction", ctypes.c_int)]


class CCInnerFace(ctypes.Structure):
    _fields_ = [("range_start", ctypes.c_int * 3), ("range_end", ctypes.c_int * 3), ("face", ctypes.c_int),
                ("direction", ctypes.c_int), ("target_start", ctypes.c_int * 3), ("target_end", ctypes.c_int * 3),
                ("target_block", ctypes.c_int), ("target_face", ctypes.c_int), ("target_direction", ctypes.c_int),
                ("src_tar", ctypes.c_int * 3), ("loop_dir", ctypes.c_int * 3), ("target_loop_dir", ctypes.c_int * 3)]


class CCClosure(ctypes.Structure):
    _fields_ = [(k, ctypes.POINTER(ctypes.c_float)) for k in
                ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4", "out_mean", "out_scale")] + \
               [(k, ctypes.c_double) for k in ("t_center", "t_scale", "t_min", "t_max")]


class CCBc(ctypes.Structure):
    _fields_ = [("label", ctypes.c_int), ("kind", ctypes.c_int), ("thermal_type", ctypes.c_int),
                ("pad", ctypes.c_int), ("t_wall", ctypes.c_double), ("density", ctypes.c_double),
                ("u", ctypes.c_double), ("v", ctypes.c_double), ("w", ctypes.c_double),
                ("pressure", ctypes.c_double), ("temperature", ctypes.c_double),
                ("yk", ctypes.c_double * MAX_SPECIES)]


EXPORTS = {
    "cc_last_error": ([], ctypes.c_char_p),
    "cc_version": ([], ctypes.c_int),
    "cc_device_count": ([ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cc_create": ([ctypes.POINTER(CCParams), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "cc_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "cc_add_block": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp,
                      ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cc_register_boundary": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(CCBoundary)],
                             ctypes.c_int),
    "cc_register_inner_face": ([ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(CCInnerFace)],
                               ctypes.c_int),
    "cc_add_boundary": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(CCBoundary)], ctypes.c_int),
    "cc_add_inner_face": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(CCInnerFace)], ctypes.c_int),
    "cc_add_bc": ([ctypes.c_void_p, ctypes.POINTER(CCBc)], ctypes.c_int),
    "cc_set_state": ([ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int], ctypes.c_int),
    "cc_init": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_step": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "cc_residual": ([ctypes.c_void_p, _dp], ctypes.c_int),
    "cc_get_state": ([ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, ctypes.c_int], ctypes.c_int),
    "cc_get_props": ([ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp], ctypes.c_int),
    "cc_last_dt": ([ctypes.c_void_p, _dp], ctypes.c_int),
    "cc_status": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint)], ctypes.c_int),
    "cc_set_stream": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "cc_get_stream": ([ctypes.c_void_p], ctypes.c_void_p),
    "cc_use_graph": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_set_renormalize": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_residual_async": ([ctypes.c_void_p, _dp], ctypes.c_int),
    "cc_set_wait_limit": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int),
    "cc_set_newton_max_iter": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_info": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cc_time_kernels": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp], ctypes.c_int),
    "cc_tuning": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _dp,
                   ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cc_set_tuning": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "cc_set_launch_mode": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_set_tile_width": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_set_closure": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "cc_use_closure": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "cc_closure_stats": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "cc_set_closure_bound": ([ctypes.c_void_p, ctypes.c_double], ctypes.c_int),
    "cc_eval_transport": ([ctypes.c_void_p, ctypes.c_int64, _dp, _dp, ctypes.c_int, _dp], ctypes.c_int),
    "cc_save_checkpoint": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "cc_load_checkpoint": ([ctypes.c_void_p, ctypes.c_char_p], ctypes.c_int),
    "cc_sync": ([ctypes.c_void_p], ctypes.c_int),
    "cc_halo_dependencies": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                              ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "cc_block_arena": ([ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64),
                        ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "cc_mlp_param_count": ([ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int64),
    "cc_mlp_workspace_bytes": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int64),
    "cc_mlp_grad": ([ctypes.c_int] * 4 + [ctypes.c_void_p] * 8, ctypes.c_int),
    "cc_mlp_adam": ([ctypes.c_int64] + [ctypes.c_void_p] * 4 + [ctypes.c_float] * 4 + [ctypes.c_int, ctypes.c_void_p],
                    ctypes.c_int),
    "cc_residual_rms_noalloc": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p],
                                ctypes.c_int),
    "cc_set_owned_blocks": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int], ctypes.c_int),
    "cc_set_exchange": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "cc_exchange_fields": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "cc_pack_points": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, _dp], ctypes.c_int),
    "cc_unpack_points": ([ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, _dp], ctypes.c_int),
    "cc_residual_sums": ([ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
}

# cc_exchange_fn: int (*)(void *user, int event, int stage, double *value)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp)
CC_EXCHANGE_STAGE, CC_EXCHANGE_DT = 0, 1

_lib = None


class CCError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Loads libcc_b200.so (built by combustioncodegpu_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CCError("libcc_b200.so not built (%s); run python -m combustioncodegpu_b200.build" % path)
    lib = ctypes.CDLL(path)
    for name, (args, res) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc):
    if rc != 0:
        raise CCError("libcc_b200 error %d: %s" % (rc, _lib.cc_last_error().decode()))


def _ptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def device_count():
    lib = load_library()
    n = ctypes.c_int(0)
    _check(lib.cc_device_count(ctypes.byref(n)))
    return n.value


def register_boundary(raw, ngg=2):
    """Boundary::register_boundary (Mesh.cpp:14-32) on a raw record."""
    lib = load_library()
    arr = (ctypes.c_int * 7)(*raw)
    out = CCBoundary()
    _check(lib.cc_register_boundary(arr, ngg, ctypes.byref(out)))
    return out


def register_inner_face(raw, ngg=2):
    """InnerFace ctor + register_boundary (Mesh.cpp:35-143) on a raw record."""
    lib = load_library()
    arr = (ctypes.c_int * 13)(*raw)
    out = CCInnerFace()
    _check(lib.cc_register_inner_face(arr, ngg, ctypes.byref(out)))
    return out


def boundary_tuple(b):
    return (tuple(b.range_start), tuple(b.range_end), b.type_label, b.face, b.direction)


def inner_face_tuple(f):
    return (tuple(f.range_start), tuple(f.range_end), f.face, f.direction, tuple(f.target_start),
            tuple(f.target_end), f.target_block, f.target_face, f.target_direction, tuple(f.src_tar),
            tuple(f.loop_dir), tuple(f.target_loop_dir))


class Parameter(dict):
    """cfd::Parameter (Parameter.h:12-67): typed key/value store with the
    reference's key names (inviscid_scheme, reconstruction, limiter,
    viscous_order, cfl, prandtl_number, schmidt_number, ngg, ...)."""

    def get_int(self, k):
        return int(self[k])

    def get_real(self, k):
        return float(self[k])

    def get_bool(self, k):
        return bool(self[k])

    def get_string(self, k):
        return str(self[k])


class Block:
    """cfd::Block (Mesh.h:109-159): extents, Jacobian, metrics and the raw
    boundary / inner-face records of the mesh files."""

    def __init__(self, dims, jac, metric, boundaries=(), inner_faces=()):
        self.mx, self.my, self.mz = (int(d) for d in dims)
        self.jac = np.ascontiguousarray(jac, dtype=np.float64)
        self.metric = np.ascontiguousarray(metric, dtype=np.float64).reshape(9, -1)
        self.boundary = [list(b) for b in boundaries]
        self.inner_face = [list(f) for f in inner_faces]

    @property
    def dims(self):
        return (self.mx, self.my, self.mz)

    def n_ghosted(self, ngg=2):
        return (self.mx + 2 * ngg) * (self.my + 2 * ngg) * (self.mz + 2 * ngg)


class Mesh(list):
    """cfd::Mesh (Mesh.h:163-232): the blocks of one process."""

    @property
    def n_block(self):
        return len(self)

    @property
    def n_grid_total(self):
        return sum(b.mx * b.my * b.mz for b in self)


def _layout(name):
    """CC_LAYOUT_FIELD_MAJOR (0) for "field", CC_LAYOUT_POINT_MAJOR (1) for "point"."""
    if name not in ("field", "point"):
        raise ValueError("layout must be 'field' or 'point'")
    return 1 if name == "point" else 0


class Field:
    """cfd::Field (Field.h:67-82): one block's state on the device."""

    def __init__(self, driver, index, block):
        self.driver, self.index, self.block = driver, index, block

    def get_state(self, layout="field"):
        """(bv, yk, cv) as FP64 host arrays: [6][Ng], [n_spec][Ng],
        [n_var][Ng] (layout "field"), or [Ng][6], [Ng][n_spec], [Ng][n_var]
        (layout "point", the reference's VectorField3D order)."""
        d = self.driver
        ng = self.block.n_ghosted(d.ngg)
        pm = _layout(layout)
        shape = (lambda nf: (ng, nf)) if pm else (lambda nf: (nf, ng))
        bv = np.empty(shape(6))
        yk = np.empty(shape(max(d.n_spec, 0)))
        cv = np.empty(shape(5 + d.n_spec))
        _check(d.lib.cc_get_state(d.ctx, self.index, _ptr(bv), _ptr(yk) if d.n_spec else None, _ptr(cv), pm))
        return bv, yk, cv

    def get_props(self):
        """(mul [Ng], conductivity [Ng], rho_D [n_spec][Ng])."""
        d = self.driver
        ng = self.block.n_ghosted(d.ngg)
        mul, cond = np.empty(ng), np.empty(ng)
        rd = np.empty((max(d.n_spec, 0), ng))
        _check(d.lib.cc_get_props(d.ctx, self.index, _ptr(mul), _ptr(cond), _ptr(rd) if d.n_spec else None))
        return mul, cond, rd

    def set_state(self, bv, yk=None, layout="field"):
        """bv (and yk) in layout "field" ([n_field][Ng]) or "point"
        ([Ng][n_field])."""
        d = self.driver
        bv = np.ascontiguousarray(bv, dtype=np.float64)
        yk = np.ascontiguousarray(yk, dtype=np.float64) if d.n_spec else None
        _check(d.lib.cc_set_state(d.ctx, self.index, _ptr(bv), _ptr(yk), _layout(layout)))


def make_params(parameter, species):
    """cc_params from a Parameter and a species dict; returns (struct, keepalive)."""
    ns = 0 if species is None else int(species["n_spec"])
    p = CCParams()
    p.n_spec = ns
    p.inviscid_scheme = parameter.get_int("inviscid_scheme")
    p.reconstruction = parameter.get_int("reconstruction")
    p.limiter = parameter.get_int("limiter")
    p.viscous_order = parameter.get_int("viscous_order")
    p.ngg = parameter.get_int("ngg")
    p.prandtl_number = parameter.get_real("prandtl_number")
    p.cfl = parameter.get_real("cfl")
    p.schmidt_number = parameter.get_real("schmidt_number")
    keep = []
    if ns:
        for name in ("mw", "t_low", "t_mid", "t_high", "low_temp_coeff", "high_temp_coeff", "LJ_potent_inv",
                     "vis_coeff", "WjDivWi_to_One4th", "sqrt_WiDivWjPl1Mul8"):
            a = np.ascontiguousarray(species[name], dtype=np.float64).ravel()
            keep.append(a)
            setattr(p, name, _ptr(a))
    return p, keep


def make_bc(d, n_spec):
    b = CCBc()
    b.label = int(d["label"])
    b.kind = int(d["kind"])
    b.thermal_type = int(d.get("thermal_type", 0))
    b.t_wall = float(d.get("t_wall", 300.0))
    for k in ("density", "u", "v", "w", "pressure", "temperature"):
        setattr(b, k, float(d.get(k, 0.0)))
    yk = np.zeros(MAX_SPECIES)
    if "yk" in d:
        yk[:n_spec] = np.asarray(d["yk"], dtype=np.float64)[:n_spec]
    for i in range(MAX_SPECIES):
        b.yk[i] = yk[i]
    return b


class Driver:
    """cfd::Driver (Driver.h:17-48) on the sm_100a path.

    Driver(parameter, mesh, species, bcs, initial_states) sets up the device
    context (Driver.cu:17-57); initialize_computation() is Driver.cu:59-97;
    simulate(n) advances n steps of SSP-RK3 (or the reference's steady
    explicit-Euler loop with scheme='steady')."""

    def __init__(self, parameter, mesh, species=None, bcs=(), states=None, precision="fp64"):
        self.lib = load_library()
        self.parameter = parameter
        self.mesh = mesh
        self.species = species
        self.n_spec = 0 if species is None else int(species["n_spec"])
        self.ngg = parameter.get_int("ngg")
        self.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        p, self._keep = make_params(parameter, species)
        ctx = ctypes.c_void_p()
        _check(self.lib.cc_create(ctypes.byref(p), ctypes.byref(ctx)))
        self.ctx = ctx
        self.field = []
        for b in mesh:
            bid = ctypes.c_int()
            _check(self.lib.cc_add_block(self.ctx, b.mx, b.my, b.mz, _ptr(b.jac), _ptr(b.metric), ctypes.byref(bid)))
            for raw in b.boundary:
                _check(self.lib.cc_add_boundary(self.ctx, bid.value, ctypes.byref(register_boundary(raw, self.ngg))))
            for raw in b.inner_face:
                _check(self.lib.cc_add_inner_face(self.ctx, bid.value,
                                                  ctypes.byref(register_inner_face(raw, self.ngg))))
            self.field.append(Field(self, bid.value, b))
        for bc in bcs:
            _check(self.lib.cc_add_bc(self.ctx, ctypes.byref(make_bc(bc, self.n_spec))))
        if states is not None:
            for f, (bv, yk) in zip(self.field, states):
                f.set_state(bv, yk)

    @classmethod
    def from_case(cls, case, precision="fp64"):
        params = Parameter(case["params"])
        mesh = Mesh(Block(b["dims"], b["jac"], b["metric"], b["boundaries"], b["inner_faces"])
                    for b in case["blocks"])
        states = [(b["bv"], b["yk"]) for b in case["blocks"]]
        return cls(params, mesh, case["params"].get("species"), case["bcs"], states, precision)

    def initialize_computation(self):
        _check(self.lib.cc_init(self.ctx, self.precision))

    def simulate(self, n_steps, scheme="rk3", residual=False):
        sch = SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
        _check(self.lib.cc_step(self.ctx, int(n_steps), sch, 1 if residual else 0))

    def residual(self):
        out = np.zeros(4)
        _check(self.lib.cc_residual(self.ctx, _ptr(out)))
        return out

    def last_dt(self):
        out = np.zeros(1)
        _check(self.lib.cc_last_dt(self.ctx, _ptr(out)))
        return float(out[0])

    def status(self):
        f = ctypes.c_uint(0)
        _check(self.lib.cc_status(self.ctx, ctypes.byref(f)))
        return f.value

    def stream(self):
        return self.lib.cc_get_stream(self.ctx)

    def set_stream(self, stream_ptr):
        _check(self.lib.cc_set_stream(self.ctx, ctypes.c_void_p(stream_ptr)))

    def set_renormalize(self, enable):
        """Y renormalisation after each update: True/False, or None for the
        precision's default (mixed on, FP64 off)."""
        _check(self.lib.cc_set_renormalize(self.ctx, -1 if enable is None else (1 if enable else 0)))

    def set_wait_limit(self, spins=None):
        """Polls of a device-side wait (after one non-blocking check) before
        the kernel gives up and sets its status bit; None restores the
        default."""
        _check(self.lib.cc_set_wait_limit(self.ctx, -1 if spins is None else int(spins)))

    def set_newton_max_iter(self, n=0):
        """Iteration cap of the temperature Newton; 0 restores the
        reference's 1000."""
        _check(self.lib.cc_set_newton_max_iter(self.ctx, int(n)))

    def use_graph(self, enable=True):
        _check(self.lib.cc_use_graph(self.ctx, 1 if enable else 0))

    def time_kernels(self, n_steps, scheme="rk3"):
        """Event-timed run without graph replay: dict of mean stage-kernel ms
        per launch, mean halo ms per stage, launches, stage+halo ms per step."""
        out = np.zeros(6)
        sch = SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
        _check(self.lib.cc_time_kernels(self.ctx, int(n_steps), sch, _ptr(out)))
        return {"stage_ms": out[0], "halo_ms": out[1], "stage_launches": int(out[2]), "step_ms": out[3],
                "faces_ms": out[4], "update_ms": out[5]}

    def sync(self):
        _check(self.lib.cc_sync(self.ctx))

    def info(self):
        n, nb, nt, nl = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_int()
        _check(self.lib.cc_info(self.ctx, ctypes.byref(n), ctypes.byref(nb), ctypes.byref(nt), ctypes.byref(nl)))
        return {"n_points": n.value, "device_bytes": nb.value, "n_tiles": nt.value, "halo_levels": nl.value}

    def tuning(self):
        """Stage-kernel configuration in use: variant ("l1" fused with L1
        stencil reads, "tma" fused with TMA-staged planes, "split" face and
        update kernels, "split-tma" the same with TMA-staged planes in the
        face kernel, "split-tma-p" on persistent CTAs, "dq-tma" a face kernel
        that differences the faces inside its tile), k-planes per tile, the
        face kernel's tile (i, j, k) in points, measured ms per stage."""
        v, kz, ms = ctypes.c_int(), ctypes.c_int(), np.zeros(1)
        tile = (ctypes.c_int * 3)()
        _check(self.lib.cc_tuning(self.ctx, ctypes.byref(v), ctypes.byref(kz), _ptr(ms), tile))
        return {"variant": VARIANTS[v.value], "kz": kz.value, "stage_ms": float(ms[0]), "tile": tuple(tile)}

    def set_tuning(self, variant="auto", kz=0, tile_j=0, tile_i=0):
        """Pin the stage-kernel configuration: variant "auto" or one of
        VARIANTS; kz k-planes per tile (0 = autotune); tile_j points along j
        of the TMA face kernels' tile (4, 8, 16; 0 = autotune); tile_i points
        along i of the "split-tma" / "split-tma-p" face tile (32, 16; 0 =
        autotune)."""
        v = (-1 if variant == "auto" else VARIANTS.index(variant)) if isinstance(variant, str) else int(variant)
        _check(self.lib.cc_set_tile_width(self.ctx, int(tile_i)))
        _check(self.lib.cc_set_tuning(self.ctx, v, int(kz), int(tile_j)))

    def set_launch_mode(self, mode="batched"):
        """"batched": one launch per stage kernel over all blocks;
        "per_block": one launch per block per kernel (the reference's way)."""
        _check(self.lib.cc_set_launch_mode(self.ctx, {"batched": 0, "per_block": 1}[mode]))

    def halo_dependencies(self):
        """(dst, src, which) int64/int64/int32 arrays: arena point src of the
        current (which 0) or previous (1) state that the halo program's final
        value of point dst is computed from (cc_halo_dependencies; host only)."""
        n = ctypes.c_int64(0)
        _check(self.lib.cc_halo_dependencies(self.ctx, None, None, None, 0, ctypes.byref(n)))
        dst = np.empty(n.value, dtype=np.int64)
        src = np.empty(n.value, dtype=np.int64)
        which = np.empty(n.value, dtype=np.int32)
        _check(self.lib.cc_halo_dependencies(self.ctx, dst.ctypes.data, src.ctypes.data, which.ctypes.data,
                                             n.value, ctypes.byref(n)))
        return dst, src, which

    def block_arena(self, block):
        """(first, count): the arena points of a block's ghosted box (cc_block_arena)."""
        first, count = ctypes.c_int64(0), ctypes.c_int64(0)
        _check(self.lib.cc_block_arena(self.ctx, int(block), ctypes.byref(first), ctypes.byref(count)))
        return first.value, count.value

    def save_checkpoint(self, path):
        """The current state, bit for bit (cc_save_checkpoint)."""
        _check(self.lib.cc_save_checkpoint(self.ctx, str(path).encode()))

    def load_checkpoint(self, path):
        """Restore a state saved by save_checkpoint into this initialised
        context (same blocks, species and precision)."""
        _check(self.lib.cc_load_checkpoint(self.ctx, str(path).encode()))

    def set_closure(self, weights):
        """Upload a learned transport closure: a dict with w1, b1, ..., w4,
        b4, out_mean, out_scale (float32 arrays) and t_center, t_scale,
        t_min, t_max (see cc_b200.h, cc_closure)."""
        keep = {k: np.ascontiguousarray(weights[k], dtype=np.float32)
                for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4", "out_mean", "out_scale")}
        fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        m = CCClosure(*(fp(keep[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4", "out_mean",
                                              "out_scale")),
                      float(weights["t_center"]), float(weights["t_scale"]), float(weights["t_min"]),
                      float(weights["t_max"]))
        _check(self.lib.cc_set_closure(self.ctx, ctypes.byref(m)))

    def use_closure(self, on=True):
        _check(self.lib.cc_use_closure(self.ctx, 1 if on else 0))

    def closure_stats(self):
        """(points evaluated by the closure kernel, exact outside the
        training hull, exact after the run-time error check)."""
        out = (ctypes.c_int64 * 3)()
        _check(self.lib.cc_closure_stats(self.ctx, out))
        return int(out[0]), int(out[1]), int(out[2])

    def set_closure_bound(self, rel_err=1e-3):
        """Relative error bound of the closure's run-time check (0: off)."""
        _check(self.lib.cc_set_closure_bound(self.ctx, float(rel_err)))

    def eval_transport(self, T, Y, mode="exact"):
        """(mu, lambda, rhoD_k) [2 + n_spec][n] of points (T [n], Y [n_spec][n])
        by the exact FP64 kernel ("exact") or the closure kernel ("closure")."""
        T = np.ascontiguousarray(T, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        out = np.empty((2 + self.n_spec, T.size))
        _check(self.lib.cc_eval_transport(self.ctx, T.size, _ptr(T), _ptr(Y), {"exact": 0, "closure": 1}[mode],
                                          _ptr(out)))
        return out

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.cc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
