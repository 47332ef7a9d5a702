"""Host-side Python mirror of the reference driver's interface to the hot path.

The reference (AMR-LBM-OpenMP-2D, Fortran 90 + OpenMP) drives its solver
from ``Main_Loop`` (AMR_Rising_2D_OMP.f90:267-377) by calling, in order,
``Determine_Min_Max_Levels``, ``Fill_Ghost_Cells_C2``,
``Phase_Field_LBM_h_g_AMR``, ``Macroscopic_Values_h_AMR``,
``Fill_Ghost_Cells_C``, ``Macroscopic_Values_g_AMR`` and
``Refine_Derefine_Mesh``. :class:`AmrLbm` exposes exactly those call sites
(same names in snake case, same meaning) over the C ABI of ``libamrlbm.so``
(``include/amrlbm.h``), whose kernels run on the B200. Every method raises
:class:`AmrLbmError` with the library's message when the status is not 0;
there is no CPU fallback: a missing library or device is an error.

Field arrays use the reference's layouts (Parameters.f90:36-37) as numpy
arrays in Fortran order: ``h, g`` (9, nx+2, ny+2), ``C`` (nx+4, ny+4),
``P, Ux, Uy`` (nx, ny).
"""
from __future__ import annotations

import ctypes as ct
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libamrlbm.so")

# status codes (include/amrlbm.h)
OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_POOL_FULL = 3
ERR_LEVEL_JUMP = 4
ERR_NAN = 5
ERR_DANGLING = 6
ERR_STATE = 7
ERR_TIMEOUT = 8
ERR_CAPACITY = 9
ERR_IO = 10
G_MRT, G_BGK = 0, 1  # collision models of g (amrlbm_set_g_collision)
FP64, FP16, BF16 = 0, 1, 2  # storage precisions of amrlbm_step (amrlbm_set_precision)

F_LEAF, F_HASLEAF, F_REFIN, F_DEREF, F_ALLOC = 1, 2, 4, 8, 16


class Params(ct.Structure):
    """``amrlbm_params`` (include/amrlbm.h)."""

    _fields_ = [
        ("nx", ct.c_int32), ("ny", ct.c_int32),
        ("nbx", ct.c_int32), ("nby", ct.c_int32),
        ("dx0", ct.c_int32),
        ("min_levels", ct.c_int32), ("max_levels", ct.c_int32),
        ("max_blks", ct.c_int32),
        ("regrid_every", ct.c_int32), ("device", ct.c_int32),
        ("rho_l", ct.c_double), ("rho_h", ct.c_double),
        ("visc_ratio", ct.c_double),
        ("bo", ct.c_double), ("ar", ct.c_double),
        ("gy", ct.c_double),
        ("w", ct.c_double), ("m0", ct.c_double),
        ("radius", ct.c_double), ("xc", ct.c_double), ("yc", ct.c_double),
        ("refin_tol", ct.c_double), ("deref_tol", ct.c_double),
        ("hydrostatic_start", ct.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Instance(ct.Structure):
    """``amrlbm_instance`` (include/amrlbm.h): one problem of a batch."""

    _fields_ = [
        ("nbx", ct.c_int32), ("nby", ct.c_int32), ("dx0", ct.c_int32), ("max_levels", ct.c_int32),
        ("rho_l", ct.c_double), ("rho_h", ct.c_double), ("visc_ratio", ct.c_double),
        ("bo", ct.c_double), ("ar", ct.c_double), ("gy", ct.c_double), ("w", ct.c_double),
        ("m0", ct.c_double), ("radius", ct.c_double), ("xc", ct.c_double), ("yc", ct.c_double),
        ("hydrostatic_start", ct.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}

    @staticmethod
    def from_params(p: "Params") -> "Instance":
        """The instance that runs the same problem as one-mesh params p."""
        return Instance(nbx=p.nbx, nby=p.nby, dx0=p.dx0, max_levels=p.max_levels, rho_l=p.rho_l,
                        rho_h=p.rho_h, visc_ratio=p.visc_ratio, bo=p.bo, ar=p.ar, gy=p.gy, w=p.w,
                        m0=p.m0, radius=p.radius, xc=p.xc, yc=p.yc,
                        hydrostatic_start=p.hydrostatic_start)

    def params(self, batch: "Params") -> "Params":
        """One-mesh params of this instance under the batch's block size,
        tolerances and regrid interval (the same problem run alone)."""
        q = Params(**batch.as_dict())
        for k in ("nbx", "nby", "dx0", "max_levels", "rho_l", "rho_h", "visc_ratio", "bo", "ar",
                  "gy", "w", "m0", "radius", "xc", "yc", "hydrostatic_start"):
            setattr(q, k, getattr(self, k))
        q.min_levels = 0
        q.max_blks = tree_blocks(q.nbx, q.nby, q.max_levels)
        return q


class Physics(ct.Structure):
    """``amrlbm_physics`` (include/amrlbm.h), D2Q9_Mod.f90:13-16."""

    _fields_ = [(k, ct.c_double) for k in
                ("w", "sigma", "beta", "kappa", "tau_l", "tau_h", "rho_l", "rho_h", "gy", "m0")]


def reference_params() -> Params:
    """The reference's compile-time configuration: nx=ny=8, L0=256, three base
    blocks stacked in y, minLevels=1, maxLevels=log2(L0/nx)=5,
    MaxBlks=6*(L0/nx)**2 (Parameters.f90:12-19); rho 0.001/1, Bo=Ar=40,
    Gy=5e-6, W=5, M0=0.03, R=L0/10 at (L0/2, L0/2), tolerances 0.002/0.001
    (AMR_Rising_2D_OMP.f90:154-158,241-259,276-277, D2Q9_Mod.f90:10)."""
    L0, nx = 256, 8
    return Params(nx=nx, ny=nx, nbx=1, nby=3, dx0=L0 // nx, min_levels=1,
                  max_levels=int(round(math.log(L0 // nx) / math.log(2.0))),
                  max_blks=6 * (L0 // nx) ** 2, regrid_every=1,
                  rho_l=0.001, rho_h=1.0, visc_ratio=100.0, bo=40.0, ar=40.0,
                  gy=0.000005, w=5.0, m0=0.03, radius=L0 / 10.0, xc=float(L0 // 2),
                  yc=float(L0 // 2), refin_tol=0.002, deref_tol=0.001)


def archimedes(eo: float, mo: float) -> float:
    """Ar = (Eo^3/Mo)^(1/4): the reference parameterises buoyancy by Bo (=Eo)
    and Ar (AMR_Rising_2D_OMP.f90:244-250)."""
    return (eo ** 3 / mo) ** 0.25


def tree_blocks(nbx: int, nby: int, levels: int) -> int:
    """Blocks of a fully refined quadtree over nbx x nby base blocks: an upper
    bound of the pool size the regrid can ever need."""
    return sum(nbx * nby * 4 ** l for l in range(levels + 1))


def bubble_params(base_x: int, base_y: int, levels: int, radius: float, xc: float,
                  yc: float, rho_ratio: float, visc_ratio: float, eo: float, mo: float,
                  w: float = 4.0, m0: float = 0.02, refin_tol: float = 1e-3,
                  deref_tol: float = 5e-4, regrid_every: int = 1, n: int = 16,
                  max_blks: int | None = None, gy: float = 0.000005,
                  hydrostatic_start: int = 1) -> Params:
    """A rising-bubble workload on a base grid of base_x x base_y cells in
    n x n blocks with `levels` refinement levels above the base (finest cell =
    1 length unit, so the base cell size is 2**levels). minLevels = 0: base
    blocks may stay leaves. hydrostatic_start=1: the start-up pressure carries
    the light phase's hydrostatic head (amrlbm_params.hydrostatic_start)."""
    assert base_x % n == 0 and base_y % n == 0
    nbx, nby = base_x // n, base_y // n
    if max_blks is None:
        max_blks = tree_blocks(nbx, nby, levels)
    return Params(nx=n, ny=n, nbx=nbx, nby=nby, dx0=2 ** levels, min_levels=0,
                  max_levels=levels, max_blks=max_blks, regrid_every=regrid_every,
                  rho_l=1.0 / rho_ratio, rho_h=1.0, visc_ratio=visc_ratio, bo=eo,
                  ar=archimedes(eo, mo), gy=gy, w=w, m0=m0, radius=radius,
                  xc=xc, yc=yc, refin_tol=refin_tol, deref_tol=deref_tol,
                  hydrostatic_start=hydrostatic_start)


def workload_small() -> Params:
    """Plain FP64 rising bubble: base grid 64x128 cells in 16x16 blocks, 2
    refinement levels (finest-equivalent 256x512), R=32 at (128,128),
    density ratio 10, viscosity ratio 10, Eo=10, Mo=1e-3, W=4, M=0.02,
    Gy=5e-6 (the reference's), hydrostatic start-up pressure, refine where
    |grad C| > 1e-3 (derefine tolerance 5e-4, half the refine tolerance as in
    the reference's 0.002/0.001), regrid every step."""
    return bubble_params(64, 128, 2, 32.0, 128.0, 128.0, 10.0, 10.0, 10.0, 1e-3,
                         w=4.0, m0=0.02, refin_tol=1e-3, deref_tol=5e-4, regrid_every=1)


# Gravity of the large workload: with Gy = 2.5e-7, D = 256 and Ar = 100 the
# product Gy*D**3/Ar**2, and with it both phases' viscosities and relaxation
# times (tau_h = 0.0614, tau_l = 0.614), equal the reference's own start-up
# bubble's (Gy = 5e-6, D = 51.2, Ar = 40; AMR_Rising_2D_OMP.f90:241-255).
# At the reference's Gy = 5e-6 the light phase's tau_l = 2.75 and it blows up
# on the dx=2 level within 2000 steps.
LARGE_GY = 2.5e-7


def workload_large() -> Params:
    """Plain FP64 rising bubble at scale: base grid 256x512 cells in 16x16
    blocks, 3 refinement levels (finest-equivalent 2048x4096), R=128 at
    (1024,512), density ratio 1000, viscosity ratio 100, Eo=10, Mo=1e-5, W=4,
    Gy=2.5e-7 (LARGE_GY), hydrostatic start-up pressure, regrid every 10
    steps (mobility and tolerances as the small workload)."""
    return bubble_params(256, 512, 3, 128.0, 1024.0, 512.0, 1000.0, 100.0, 10.0, 1e-5,
                         w=4.0, m0=0.02, refin_tol=1e-3, deref_tol=5e-4, regrid_every=10,
                         gy=LARGE_GY)


# Lattice limits of a batch instance: the relaxation times of both phases
# and the velocity scale sqrt(Gy D) (lattice Mach number sqrt(3) U)
TAU_RANGE = (0.02, 2.0)
U_SCALE = 0.01


def batch_instances(count: int = 256, seed: int = 20261203, n: int = 16) -> list:
    """Seeded batch of uneven rising-bubble problems: base grid uniform in
    {64x128, 128x256, 256x512} cells, 2 or 3 refinement levels (finest cell 1),
    R uniform in [16, 96] finest cells (centred in x, at a quarter of the
    height), density ratio log-uniform in [10, 1000], Eo uniform in [1, 50],
    Mo log-uniform in [1e-6, 1e-2]; viscosity ratio min(density ratio, 100),
    W 4, M0 0.02, hydrostatic start. Gy is set per instance for a velocity
    scale sqrt(Gy D) = U_SCALE; an instance whose relaxation times
    3 mu/rho leave TAU_RANGE at that gravity cannot be run on the lattice and is
    drawn again from the same stream."""
    import numpy as np
    rng = np.random.default_rng(seed)
    bases = [(64, 128), (128, 256), (256, 512)]
    out = []
    while len(out) < count:
        bx, by = bases[int(rng.integers(0, 3))]
        levels = int(rng.integers(2, 4))
        radius = float(rng.uniform(16.0, 96.0))
        ratio = float(10.0 ** rng.uniform(1.0, 3.0))
        eo = float(rng.uniform(1.0, 50.0))
        mo = float(10.0 ** rng.uniform(-6.0, -2.0))
        width, height = bx * 2 ** levels, by * 2 ** levels
        if 2.5 * radius > width or 2.5 * radius > height / 4.0:
            continue  # the bubble must fit the domain with room to rise
        D = 2.0 * radius
        gy = U_SCALE ** 2 / D
        visc = min(ratio, 100.0)
        ar = archimedes(eo, mo)
        rho_l, rho_h = 1.0 / ratio, 1.0
        muh = (gy * rho_h * (rho_h - rho_l) * D ** 3) ** 0.5 / ar
        tau_h, tau_l = 3.0 * muh / rho_h, 3.0 * (muh / visc) / rho_l
        if not (TAU_RANGE[0] <= tau_h <= TAU_RANGE[1] and TAU_RANGE[0] <= tau_l <= TAU_RANGE[1]):
            continue
        out.append(Instance(nbx=bx // n, nby=by // n, dx0=2 ** levels, max_levels=levels,
                            rho_l=rho_l, rho_h=rho_h, visc_ratio=visc, bo=eo, ar=ar, gy=gy,
                            w=4.0, m0=0.02, radius=radius, xc=width / 2.0, yc=height / 4.0,
                            hydrostatic_start=1))
    return out


def batch_params(n: int = 16, max_blks: int = 200000, regrid_every: int = 10) -> Params:
    """Batch-wide params: block size, pool size, tolerances, regrid interval.
    Refinement tolerance 3e-4 (derefinement 1.5e-4): at 1e-3 the finest level
    ends a few cells inside the interface, and in the seeded 256-problem batch
    instance 121 (density ratio 236, Eo 22) grows a light-phase instability at
    a coarse-fine corner inside its bubble before step 1400."""
    return Params(nx=n, ny=n, nbx=1, nby=1, dx0=1, min_levels=0, max_levels=0,
                  max_blks=max_blks, regrid_every=regrid_every, refin_tol=3e-4, deref_tol=1.5e-4,
                  rho_l=0.1, rho_h=1.0, visc_ratio=10.0, bo=10.0, ar=30.0, gy=5e-6, w=4.0,
                  m0=0.02, radius=16.0, xc=0.0, yc=0.0)


class AmrLbmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"amrlbm status {status}: {message}")
        self.status = status


_lib = None


def load_library(path: str | None = None):
    """Loads libamrlbm.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise AmrLbmError(ERR_STATE, f"{p} not built (run make in {_HERE})")
    lib = ct.CDLL(p)
    i32p = ct.POINTER(ct.c_int32)
    dp = ct.POINTER(ct.c_double)
    fp = ct.POINTER(ct.c_float)
    u8p = ct.POINTER(ct.c_uint8)
    vp = ct.c_void_p
    sig = {
        "amrlbm_default_params": (None, [ct.POINTER(Params)]),
        "amrlbm_derive_physics": (ct.c_int, [ct.POINTER(Params), ct.POINTER(Physics)]),
        "amrlbm_create": (ct.c_int, [ct.POINTER(Params), ct.POINTER(vp)]),
        "amrlbm_destroy": (ct.c_int, [vp]),
        "amrlbm_set_physics": (ct.c_int, [vp, ct.POINTER(Physics)]),
        "amrlbm_set_g_collision": (ct.c_int, [vp, ct.c_int32]),
        "amrlbm_set_wait_test": (ct.c_int, [vp, ct.c_int32, ct.c_int32]),
        "amrlbm_set_precision": (ct.c_int, [vp, ct.c_int32]),
        "amrlbm_get_fill_order": (ct.c_int, [vp, i32p]),
        "amrlbm_set_launch": (ct.c_int, [vp, ct.c_int32]),
        "amrlbm_set_bubbles": (ct.c_int, [vp, ct.c_int32, dp]),
        "amrlbm_block_features": (ct.c_int, [vp, ct.c_int32, i32p, ct.c_float, fp]),
        "amrlbm_set_regrid_net": (ct.c_int, [vp, vp, ct.c_float, ct.c_float]),
        "amrlbm_regrid_stats": (ct.c_int, [vp, ct.POINTER(ct.c_int64)]),
        "amrlbm_forecast_blocks": (ct.c_int, [vp, ct.c_int32, i32p, fp]),
        "amrlbm_net_create": (ct.c_int, [ct.c_uint64, ct.c_int32, ct.POINTER(vp)]),
        "amrlbm_net_destroy": (ct.c_int, [vp]),
        "amrlbm_net_param_count": (ct.c_int32, []),
        "amrlbm_net_last_error": (ct.c_char_p, [vp]),
        "amrlbm_net_get": (ct.c_int, [vp, fp]),
        "amrlbm_net_set": (ct.c_int, [vp, fp]),
        "amrlbm_net_forward": (ct.c_int, [vp, ct.c_int32, fp, fp]),
        "amrlbm_net_gradient": (ct.c_int, [vp, ct.c_int32, fp, fp, ct.c_float,
                                           ct.POINTER(ct.c_float), fp]),
        "amrlbm_net_train_step": (ct.c_int, [vp, ct.c_int32, fp, fp, ct.c_float, ct.c_float,
                                             ct.POINTER(ct.c_float)]),
        "amrlbm_net_selftest_gemm": (ct.c_int, [ct.c_int32, ct.c_int32, ct.c_int32,
                                                ct.POINTER(ct.c_uint16), ct.POINTER(ct.c_uint16),
                                                fp]),
        "amrlbm_create_batch": (ct.c_int, [ct.POINTER(Params), ct.c_int32, ct.POINTER(Instance),
                                           ct.POINTER(vp)]),
        "amrlbm_get_instances": (ct.c_int, [vp, i32p]),
        "amrlbm_diag_instances": (ct.c_int, [vp, dp]),
        "amrlbm_last_error": (ct.c_char_p, [vp]),
        "amrlbm_device_bytes": (ct.c_int64, [vp]),
        "amrlbm_get_counts": (ct.c_int, [vp, i32p]),
        "amrlbm_set_level_range": (ct.c_int, [vp, ct.c_int32, ct.c_int32]),
        "amrlbm_set_topology": (ct.c_int, [vp, ct.c_int32, i32p, i32p, i32p, i32p, i32p,
                                           i32p, i32p, i32p, u8p, ct.c_int32, i32p,
                                           ct.c_int32]),
        "amrlbm_get_topology": (ct.c_int, [vp, i32p, i32p, i32p, i32p, i32p, i32p, i32p,
                                           i32p, u8p, i32p, i32p]),
        "amrlbm_get_neighbours": (ct.c_int, [vp, i32p]),
        "amrlbm_get_leaves": (ct.c_int, [vp, i32p]),
        "amrlbm_upload_block": (ct.c_int, [vp, ct.c_int32, dp, dp, dp, dp, dp, dp]),
        "amrlbm_download_block": (ct.c_int, [vp, ct.c_int32, dp, dp, dp, dp, dp, dp]),
        "amrlbm_upload_fields": (ct.c_int, [vp, ct.c_int32, i32p, dp, dp, dp, dp, dp, dp]),
        "amrlbm_download_fields": (ct.c_int, [vp, ct.c_int32, i32p, dp, dp, dp, dp, dp, dp]),
        "amrlbm_get_block_error": (ct.c_int, [vp, dp]),
        "amrlbm_init_rising_bubble": (ct.c_int, [vp]),
        "amrlbm_init_fields": (ct.c_int, [vp]),
        "amrlbm_min_max_levels": (ct.c_int, [vp, i32p, i32p]),
        "amrlbm_fill_ghost_c2": (ct.c_int, [vp]),
        "amrlbm_phase_field_step": (ct.c_int, [vp]),
        "amrlbm_macro_h": (ct.c_int, [vp]),
        "amrlbm_fill_ghost_c": (ct.c_int, [vp]),
        "amrlbm_macro_g": (ct.c_int, [vp]),
        "amrlbm_regrid": (ct.c_int, [vp, ct.c_double, ct.c_double]),
        "amrlbm_step": (ct.c_int, [vp, ct.c_int32]),
        "amrlbm_sync": (ct.c_int, [vp]),
        "amrlbm_diag": (ct.c_int, [vp, dp]),
        "amrlbm_write_tecplot": (ct.c_int, [vp, ct.c_char_p, ct.c_int32]),
        "amrlbm_timer_start": (ct.c_int, [vp]),
        "amrlbm_timer_stop": (ct.c_int, [vp, ct.POINTER(ct.c_float)]),
        "amrlbm_profile_enable": (ct.c_int, [vp, ct.c_int32]),
        "amrlbm_profile_read": (ct.c_int, [vp, ct.c_int32, dp, ct.POINTER(ct.c_int64),
                                           ct.POINTER(ct.c_int64)]),
        "amrlbm_launch_count": (ct.c_int64, [vp]),
        "amrlbm_flush_l2": (ct.c_int, [vp]),
        "amrlbm_selftest_division": (ct.c_int, [ct.c_uint64, ct.c_uint64, ct.c_double,
                                                ct.POINTER(ct.c_uint64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols() -> list[str]:
    """Names of every entry point declared in include/amrlbm.h."""
    hdr = os.path.join(_HERE, "..", "include", "amrlbm.h")
    import re
    names = []
    with open(hdr) as f:
        for line in f:
            m = re.match(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(amrlbm_\w+)\s*\(", line)
            if m:
                names.append(m.group(1))
    return names


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ct.POINTER(ctype))


class AmrLbm:
    """One device-resident block pool, driven like the reference's Main_Loop."""

    def __init__(self, params: Params, lib=None, instances=None):
        """One mesh (params), or a batch of independent problems (instances:
        a list of Instance; params then gives block size, pool size,
        tolerances and regrid interval, amrlbm_create_batch)."""
        self.lib = lib or load_library()
        self.params = params
        self.nx, self.ny = params.nx, params.ny
        self.instances = list(instances) if instances is not None else None
        ctx = ct.c_void_p()
        if self.instances is None:
            st = self.lib.amrlbm_create(ct.byref(params), ct.byref(ctx))
        else:
            arr = (Instance * len(self.instances))(*self.instances)
            st = self.lib.amrlbm_create_batch(ct.byref(params), len(self.instances), arr,
                                              ct.byref(ctx))
        if st != 0:
            raise AmrLbmError(st, "amrlbm_create failed (is a B200 visible?)")
        self.ctx = ctx

    # -- plumbing ---------------------------------------------------------
    def _check(self, st):
        if st != 0:
            msg = self.lib.amrlbm_last_error(self.ctx)
            raise AmrLbmError(st, msg.decode() if msg else "")
        return st

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.amrlbm_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def hshape(self):
        return (9, self.nx + 2, self.ny + 2)

    @property
    def cshape(self):
        return (self.nx + 4, self.ny + 4)

    @property
    def pshape(self):
        return (self.nx, self.ny)

    # -- driver ------------------------------------------------------------
    def initialize_rising_bubble(self):
        """AMR_LBM_Rising_Bubble start-up (AMR_Rising_2D_OMP.f90:49-67)."""
        self._check(self.lib.amrlbm_init_rising_bubble(self.ctx))

    def initialize_fields(self):
        """Initialize_AMR_Rising_Bubble (AMR_Rising_2D_OMP.f90:142-231)."""
        self._check(self.lib.amrlbm_init_fields(self.ctx))

    def set_physics(self, phys: Physics):
        self._check(self.lib.amrlbm_set_physics(self.ctx, ct.byref(phys)))

    def set_precision(self, precision):
        """FP64 (bit for bit with the reference), FP16 or BF16 storage of the
        populations for main_loop (amrlbm_set_precision); also "fp64",
        "fp16", "bf16"."""
        if isinstance(precision, str):
            precision = {"fp64": FP64, "fp16": FP16, "bf16": BF16}[precision.lower()]
        self._check(self.lib.amrlbm_set_precision(self.ctx, int(precision)))

    def set_bubbles(self, xyr):
        """Several bubbles (rows x, y, R) for the start-up (amrlbm_set_bubbles)."""
        a = np.ascontiguousarray(np.asarray(xyr, dtype=np.float64).reshape(-1, 3))
        self._check(self.lib.amrlbm_set_bubbles(self.ctx, len(a), _ptr(a, ct.c_double)))

    def block_features(self, ids, horizon: float = 16.0):
        """The forecaster's samples of blocks ids (amrlbm_block_features):
        float32 [n][4][18][18]."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        x = np.zeros((len(ids), NET_CHANNELS, NET_TILE, NET_TILE), dtype=np.float32)
        self._check(self.lib.amrlbm_block_features(self.ctx, len(ids), _ptr(ids, ct.c_int32),
                                                   horizon, _ptr(x, ct.c_float)))
        return x

    def set_regrid_net(self, net, horizon: float = 16.0, threshold: float = 0.5):
        """Learned regrid with the forecaster `net` (a Net; None: the
        criterion alone), amrlbm_set_regrid_net."""
        self._net = net
        self._check(self.lib.amrlbm_set_regrid_net(self.ctx, net.h if net else None, horizon,
                                                   threshold))

    def forecast_blocks(self, ids):
        """Logits of the attached forecaster on blocks ids by the fused kernel
        of the learned regrid (amrlbm_forecast_blocks)."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        z = np.zeros(len(ids), dtype=np.float32)
        self._check(self.lib.amrlbm_forecast_blocks(self.ctx, len(ids), _ptr(ids, ct.c_int32),
                                                    _ptr(z, ct.c_float)))
        return z

    def regrid_stats(self):
        """amrlbm_regrid_stats since the start-up: regrids, leaves forecast,
        leaves the criterion flagged (escapes), flagged ones the forecast
        missed, forecast ones not flagged."""
        a = (ct.c_int64 * 5)()
        self._check(self.lib.amrlbm_regrid_stats(self.ctx, a))
        return dict(zip(("regrids", "forecast", "flagged", "missed", "extra"), list(a)))

    def set_launch(self, ctas_per_sm: int = 0):
        """At most ctas_per_sm CTAs per SM for the mixed-precision kernels
        (0: as many as fit; amrlbm_set_launch)."""
        self._check(self.lib.amrlbm_set_launch(self.ctx, int(ctas_per_sm)))

    def fill_order(self):
        """Which ghost fills of the current mesh need level order
        (amrlbm_get_fill_order): dict c2, c1, hg -> bool."""
        a = np.zeros(3, dtype=np.int32)
        self._check(self.lib.amrlbm_get_fill_order(self.ctx, _ptr(a, ct.c_int32)))
        return dict(zip(("c2", "c1", "hg"), (bool(v) for v in a)))

    def set_wait_test(self, spin_limit: int = 0, hold_block: int = 0):
        """Failure-detection hook of the level-ordered fills' bounded flag
        waits (amrlbm_set_wait_test); (0, 0) restores normal operation."""
        self._check(self.lib.amrlbm_set_wait_test(self.ctx, int(spin_limit), int(hold_block)))

    def set_g_collision(self, model: int):
        """G_MRT (MRT_Collision_AMR, the reference's) or G_BGK
        (BGK_Collision_AMR, commented out in the reference at
        LBM_Subroutines.f90:180)."""
        self._check(self.lib.amrlbm_set_g_collision(self.ctx, int(model)))

    # -- Main_Loop call sites ---------------------------------------------
    def determine_min_max_levels(self):
        lo, hi = ct.c_int32(), ct.c_int32()
        self._check(self.lib.amrlbm_min_max_levels(self.ctx, ct.byref(lo), ct.byref(hi)))
        return lo.value, hi.value

    def set_level_range(self, lmin, lmax):
        self._check(self.lib.amrlbm_set_level_range(self.ctx, lmin, lmax))

    def fill_ghost_cells_c2(self):
        self._check(self.lib.amrlbm_fill_ghost_c2(self.ctx))

    def phase_field_lbm_h_g(self):
        self._check(self.lib.amrlbm_phase_field_step(self.ctx))

    def macroscopic_values_h(self):
        self._check(self.lib.amrlbm_macro_h(self.ctx))

    def fill_ghost_cells_c(self):
        self._check(self.lib.amrlbm_fill_ghost_c(self.ctx))

    def macroscopic_values_g(self):
        self._check(self.lib.amrlbm_macro_g(self.ctx))

    def refine_derefine_mesh(self, refin_tol=None, deref_tol=None):
        rt = self.params.refin_tol if refin_tol is None else refin_tol
        dt = self.params.deref_tol if deref_tol is None else deref_tol
        self._check(self.lib.amrlbm_regrid(self.ctx, rt, dt))

    def main_loop(self, nsteps: int):
        """nsteps iterations of the Main_Loop body (fused, graph-captured)."""
        self._check(self.lib.amrlbm_step(self.ctx, nsteps))

    def sync(self):
        self._check(self.lib.amrlbm_sync(self.ctx))

    def tecplot_cell_center(self, path, t: int):
        """TecPlot_CellCenter (TecPlot_ASCII.f90:2-86): the leaves as one
        FE-quadrilateral zone in the reference's ASCII layout, written to
        `path`; t is the time step T of the zone title."""
        self._check(self.lib.amrlbm_write_tecplot(self.ctx, os.fsencode(path), int(t)))

    def output(self):
        """Output (AMR_Rising_2D_OMP.f90:456-489) + bubble centroid/rise velocity."""
        out = np.zeros(8)
        self._check(self.lib.amrlbm_diag(self.ctx, _ptr(out, ct.c_double)))
        return dict(zip(("mass", "rho_min", "rho_max", "u_max", "bubble_volume",
                         "y_centroid", "rise_velocity", "phase_volume"), out.tolist()))

    def output_instances(self):
        """Output per instance of a batch (amrlbm_diag_instances): a list of
        dicts as output()."""
        ni = len(self.instances) if self.instances else 1
        out = np.zeros(8 * ni)
        self._check(self.lib.amrlbm_diag_instances(self.ctx, _ptr(out, ct.c_double)))
        keys = ("mass", "rho_min", "rho_max", "u_max", "bubble_volume", "y_centroid",
                "rise_velocity", "phase_volume")
        return [dict(zip(keys, out[8 * i:8 * i + 8].tolist())) for i in range(ni)]

    def block_instances(self):
        """Instance (0-based) of blocks 1..Nblks."""
        n = self.counts()["nblks"]
        a = np.zeros(max(n, 1), dtype=np.int32)
        self._check(self.lib.amrlbm_get_instances(self.ctx, _ptr(a, ct.c_int32)))
        return a[:n]

    # -- state -------------------------------------------------------------
    def counts(self):
        c = np.zeros(5, dtype=np.int32)
        self._check(self.lib.amrlbm_get_counts(self.ctx, _ptr(c, ct.c_int32)))
        return dict(zip(("nblks", "nleaf", "kk", "level_min", "level_max"), c.tolist()))

    def topology(self):
        n = self.counts()["nblks"]
        i32 = lambda k=1: np.zeros(n * k, dtype=np.int32)
        t = dict(level=i32(), dx=i32(), bi=i32(), bj=i32(), parent=i32(), child=i32(4),
                 nbr_owner=i32(8), nbr_slot=i32(8), flags=np.zeros(n, dtype=np.uint8))
        nfree = ct.c_int32()
        fl = np.zeros(self.params.max_blks // 4 + 1, dtype=np.int32)
        self._check(self.lib.amrlbm_get_topology(
            self.ctx, *[_ptr(t[k], ct.c_int32) for k in
                        ("level", "dx", "bi", "bj", "parent", "child", "nbr_owner",
                         "nbr_slot")],
            _ptr(t["flags"], ct.c_uint8), ct.byref(nfree), _ptr(fl, ct.c_int32)))
        t["free_list"] = fl[: nfree.value].copy()
        t["child"] = t["child"].reshape(n, 4)
        t["nbr_owner"] = t["nbr_owner"].reshape(n, 8)
        t["nbr_slot"] = t["nbr_slot"].reshape(n, 8)
        return t

    def set_topology(self, t, kk):
        n = len(t["level"])
        c = lambda a: np.ascontiguousarray(a, dtype=np.int32).ravel()
        arrs = [c(t[k]) for k in ("level", "dx", "bi", "bj", "parent", "child",
                                  "nbr_owner", "nbr_slot")]
        flags = np.ascontiguousarray(t["flags"], dtype=np.uint8)
        fl = c(t["free_list"]) if len(t["free_list"]) else np.zeros(1, np.int32)
        self._check(self.lib.amrlbm_set_topology(
            self.ctx, n, *[_ptr(a, ct.c_int32) for a in arrs], _ptr(flags, ct.c_uint8),
            len(t["free_list"]), _ptr(fl, ct.c_int32), kk))

    def neighbours(self):
        n = self.counts()["nblks"]
        a = np.zeros(8 * n, dtype=np.int32)
        self._check(self.lib.amrlbm_get_neighbours(self.ctx, _ptr(a, ct.c_int32)))
        return a.reshape(n, 8)

    def leaves(self):
        n = self.counts()["nleaf"]
        a = np.zeros(max(n, 1), dtype=np.int32)
        self._check(self.lib.amrlbm_get_leaves(self.ctx, _ptr(a, ct.c_int32)))
        return a[:n]

    def block_errors(self):
        n = self.counts()["nblks"]
        a = np.zeros(n)
        self._check(self.lib.amrlbm_get_block_error(self.ctx, _ptr(a, ct.c_double)))
        return a

    def download_block(self, bid):
        h = np.zeros(self.hshape, order="F")
        g = np.zeros(self.hshape, order="F")
        C = np.zeros(self.cshape, order="F")
        P = np.zeros(self.pshape, order="F")
        Ux = np.zeros(self.pshape, order="F")
        Uy = np.zeros(self.pshape, order="F")
        self._check(self.lib.amrlbm_download_block(
            self.ctx, bid, *[_ptr(a, ct.c_double) for a in (h, g, C, P, Ux, Uy)]))
        return dict(h=h, g=g, C=C, P=P, Ux=Ux, Uy=Uy)

    def upload_block(self, bid, h=None, g=None, C=None, P=None, Ux=None, Uy=None):
        f = lambda a: None if a is None else np.asfortranarray(a, dtype=np.float64)
        arrs = [f(a) for a in (h, g, C, P, Ux, Uy)]
        self._check(self.lib.amrlbm_upload_block(
            self.ctx, bid, *[_ptr(a, ct.c_double) for a in arrs]))

    def download_fields(self, ids, out=None):
        """Fields of blocks `ids` as flat per-block records (n, size) in the
        reference's column-major layouts; reshape a record with order="F".
        `out`: arrays to fill (C-contiguous float64 of those shapes, e.g. in
        page-locked memory), else new ones."""
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        n = len(ids)
        hs = int(np.prod(self.hshape))
        cs = int(np.prod(self.cshape))
        ps = int(np.prod(self.pshape))
        if out is None:
            out = dict(h=np.zeros((n, hs)), g=np.zeros((n, hs)), C=np.zeros((n, cs)),
                       P=np.zeros((n, ps)), Ux=np.zeros((n, ps)), Uy=np.zeros((n, ps)))
        want = dict(h=hs, g=hs, C=cs, P=ps, Ux=ps, Uy=ps)
        for k, sz in want.items():
            a = out[k]
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (n, sz):
                raise ValueError(f"out[{k!r}] must be C-contiguous float64 of shape {(n, sz)}")
        self._check(self.lib.amrlbm_download_fields(
            self.ctx, n, _ptr(ids, ct.c_int32),
            *[_ptr(out[k], ct.c_double) for k in ("h", "g", "C", "P", "Ux", "Uy")]))
        return out

    def upload_fields(self, ids, fields):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        arrs = [None if fields.get(k) is None else np.ascontiguousarray(fields[k], np.float64)
                for k in ("h", "g", "C", "P", "Ux", "Uy")]
        self._check(self.lib.amrlbm_upload_fields(
            self.ctx, len(ids), _ptr(ids, ct.c_int32), *[_ptr(a, ct.c_double) for a in arrs]))

    # -- timing ------------------------------------------------------------
    def timer_start(self):
        self._check(self.lib.amrlbm_timer_start(self.ctx))

    def timer_stop(self) -> float:
        ms = ct.c_float()
        self._check(self.lib.amrlbm_timer_stop(self.ctx, ct.byref(ms)))
        return ms.value

    def profile(self, enable: bool):
        self._check(self.lib.amrlbm_profile_enable(self.ctx, 1 if enable else 0))

    def profile_read(self, kernel: int = 0):
        t = ct.c_double()
        n = ct.c_int64()
        cells = ct.c_int64()
        self._check(self.lib.amrlbm_profile_read(self.ctx, kernel, ct.byref(t), ct.byref(n),
                                                 ct.byref(cells)))
        return t.value, n.value, cells.value

    def launch_count(self) -> int:
        return int(self.lib.amrlbm_launch_count(self.ctx))

    def flush_l2(self):
        self._check(self.lib.amrlbm_flush_l2(self.ctx))

    def device_bytes(self) -> int:
        return int(self.lib.amrlbm_device_bytes(self.ctx))


# ---------------------------------------------------------------------------
# Autotuner of the batched mixed-precision step: block size (8x8 or 16x16
# cells, i.e. 2 or 8 warps per CTA) and CTAs per SM, timed on the batch
# itself.

def rescale_instances(instances, n_from: int, n_to: int):
    """The same problems described in n_to x n_to blocks."""
    out = []
    for i in instances:
        d = i.as_dict()
        assert (i.nbx * n_from) % n_to == 0 and (i.nby * n_from) % n_to == 0
        d["nbx"], d["nby"] = i.nbx * n_from // n_to, i.nby * n_from // n_to
        out.append(Instance(**d))
    return out


def time_intervals(sim: "AmrLbm", intervals: int, inner: int) -> float:
    """Leaf-cell updates per second (millions) over `intervals` regrid
    intervals, device-timed with the L2 flushed before each."""
    c0 = sim.profile_read(0)[2]
    ms = 0.0
    for _ in range(intervals):
        sim.flush_l2()
        sim.sync()
        sim.timer_start()
        sim.main_loop(inner)
        ms += sim.timer_stop()
    return (sim.profile_read(0)[2] - c0) / (ms / 1e3) / 1e6


def autotune(instances, precision="fp16", block_sizes=(16, 8), ctas=(0, 1, 2, 3, 4),
             n_from: int = 16, max_blks: int = 0, warmup: int = 2, intervals: int = 3,
             regrid_every: int = 10):
    """Times the batch of `instances` (given in n_from x n_from blocks) for
    every block size and CTA-per-SM cap, returns (best, table): best =
    {"block": n, "ctas_per_sm": c, "mlups": v}, table = list of those for
    every candidate that ran."""
    table = []
    for n in block_sizes:
        insts = rescale_instances(instances, n_from, n)
        mb = max_blks or 4 * sum(i.nbx * i.nby for i in insts) + 4096
        try:
            sim = AmrLbm(batch_params(n=n, max_blks=mb, regrid_every=regrid_every),
                         instances=insts)
        except AmrLbmError:
            continue
        try:
            sim.initialize_rising_bubble()
            sim.set_precision(precision)
            for c in ctas:
                sim.set_launch(c)
                for _ in range(warmup):
                    sim.main_loop(regrid_every)
                table.append({"block": n, "ctas_per_sm": c,
                              "mlups": time_intervals(sim, intervals, regrid_every)})
        finally:
            sim.close()
    best = max(table, key=lambda r: r["mlups"]) if table else None
    return best, table


# ---------------------------------------------------------------------------
# The refine-flag forecaster of the learned regrid (amrlbm_net_*).
NET_CHANNELS, NET_TILE = 4, 18


class Net:
    """The convolutional refine-flag forecaster: forward, gradient, Adam
    steps on BF16 tensor cores (amrlbm_net_*). Samples are float32 arrays
    [n][NET_CHANNELS][NET_TILE][NET_TILE], labels float32 in {0, 1}."""

    def __init__(self, seed: int = 0, max_batch: int = 512, lib=None):
        self.lib = lib or load_library()
        self.max_batch = max_batch
        h = ct.c_void_p()
        st = self.lib.amrlbm_net_create(seed, max_batch, ct.byref(h))
        if st != 0:
            raise AmrLbmError(st, "amrlbm_net_create failed (is a B200 visible?)")
        self.h = h
        self.nparam = int(self.lib.amrlbm_net_param_count())

    def _check(self, st):
        if st != 0:
            raise AmrLbmError(st, self.lib.amrlbm_net_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.amrlbm_net_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _f(a):
        return np.ascontiguousarray(a, dtype=np.float32)

    def params(self):
        p = np.zeros(self.nparam, dtype=np.float32)
        self._check(self.lib.amrlbm_net_get(self.h, _ptr(p, ct.c_float)))
        return p

    def set_params(self, p):
        p = self._f(p)
        assert p.size == self.nparam
        self._check(self.lib.amrlbm_net_set(self.h, _ptr(p, ct.c_float)))

    def forward(self, x):
        x = self._f(x)
        out = np.zeros(len(x), dtype=np.float32)
        for i in range(0, len(x), self.max_batch):
            xb = np.ascontiguousarray(x[i:i + self.max_batch])
            ob = np.zeros(len(xb), dtype=np.float32)
            self._check(self.lib.amrlbm_net_forward(self.h, len(xb), _ptr(xb, ct.c_float),
                                                    _ptr(ob, ct.c_float)))
            out[i:i + len(xb)] = ob
        return out

    def gradient(self, x, y, pos_weight=1.0):
        x, y = self._f(x), self._f(y)
        loss = ct.c_float()
        g = np.zeros(self.nparam, dtype=np.float32)
        self._check(self.lib.amrlbm_net_gradient(self.h, len(x), _ptr(x, ct.c_float),
                                                 _ptr(y, ct.c_float), pos_weight, ct.byref(loss),
                                                 _ptr(g, ct.c_float)))
        return loss.value, g

    def train_step(self, x, y, lr=1e-3, pos_weight=1.0):
        x, y = self._f(x), self._f(y)
        loss = ct.c_float()
        self._check(self.lib.amrlbm_net_train_step(self.h, len(x), _ptr(x, ct.c_float),
                                                   _ptr(y, ct.c_float), pos_weight, lr,
                                                   ct.byref(loss)))
        return loss.value


# ---------------------------------------------------------------------------
# The learned-regrid workload: several bubbles in one domain.

def random_bubbles(count: int, rmin: float, rmax: float, width: float, height: float,
                   seed: int, margin: float = 8.0, ymax_frac: float = 0.5):
    """count non-overlapping bubbles (rows x, y, R), R uniform in [rmin, rmax],
    centres uniform in the domain's lower ymax_frac, `margin` cells apart
    and from the walls (periodic in x)."""
    rng = np.random.default_rng(seed)
    out = []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > 100000:
            raise ValueError("bubbles do not fit")
        R = float(rng.uniform(rmin, rmax))
        x = float(rng.uniform(0.0, width))
        y = float(rng.uniform(R + margin, ymax_frac * height - R - margin))
        ok = True
        for (x2, y2, R2) in out:
            dxp = min(abs(x - x2), width - abs(x - x2))
            if (dxp ** 2 + (y - y2) ** 2) ** 0.5 < R + R2 + margin:
                ok = False
                break
        if ok:
            out.append((x, y, R))
    return np.array(out)


def learned_workload(base_x: int = 512, base_y: int = 1024, levels: int = 3, count: int = 8,
                     seed: int = 20261205, rmin: float = 32.0, rmax: float = 128.0,
                     regrid_every: int = 32, rho_ratio: float = 1000.0,
                     visc_ratio: float = 100.0, eo: float = 20.0, ar: float = 40.0,
                     gy: float | None = None, refin_tol: float = 3e-4,
                     deref_tol: float = 1.5e-4):
    """Learned regrid: base grid base_x x base_y in 16x16 blocks with `levels`
    refinement levels, `count` non-overlapping bubbles R in [rmin, rmax]; by
    default density ratio 1000, viscosity ratio 100, Eo 20, Ar 40 (the
    reference's), Gy such that Gy D^3 / Ar^2 with D = 128 equals the reference
    start-up bubble's (as LARGE_GY does), hydrostatic start. Refinement
    tolerance 3e-4: at 1e-3 the finest level ends about 6 cells inside a
    bubble's interface, and the light phase blows up at a corner where a
    coarser block inside the bubble meets three finer ones (R = 58: about
    step 1750, with a regrid every 10 steps or every 32). Returns
    (params, bubbles)."""
    W, H = base_x * 2 ** levels, base_y * 2 ** levels
    bubbles = random_bubbles(count, rmin, rmax, W, H, seed)
    if gy is None:
        gy = 5e-6 * 51.2 ** 3 / 40.0 ** 2 * ar ** 2 / 128.0 ** 3
    p = bubble_params(base_x, base_y, levels, float(bubbles[0, 2]), float(bubbles[0, 0]),
                      float(bubbles[0, 1]), rho_ratio, visc_ratio, eo, eo ** 3 / ar ** 4,
                      regrid_every=regrid_every, gy=gy, refin_tol=refin_tol, deref_tol=deref_tol)
    p.ar = ar
    return p, bubbles


def collect_samples(sim: "AmrLbm", regrids: int, horizon: int = 16, keep_far: float = 0.1,
                    seed: int = 0):
    """Samples of the forecaster from a run of `sim` whose regrid interval is
    2*horizon: at each regrid (step t), the samples of the leaves that may
    still refine, labelled with the reference's criterion at step t + horizon
    (no regrid in between, so the blocks are the same). Leaves with nothing
    near an interface (every cell's error term below a tenth of the tolerance
    and no flag) are kept with probability keep_far. Returns (x, y, counts)."""
    rng = np.random.default_rng(seed)
    R = sim.params.regrid_every
    assert R == 2 * horizon
    xs, ys = [], []
    seen = pos = 0
    for _ in range(regrids):
        t = sim.topology()
        leaves = sim.leaves()
        lv = t["level"][leaves - 1]
        if sim.instances:  # each instance's own level count
            inst = sim.block_instances()
            maxlv = np.array([i.max_levels for i in sim.instances])[inst[leaves - 1]]
        else:
            maxlv = sim.params.max_levels
        cand = leaves[lv < maxlv]
        x = sim.block_features(cand, float(horizon))
        sim.main_loop(horizon)
        err = sim.block_errors()
        y = (err[cand - 1] > sim.params.refin_tol).astype(np.float32)
        sim.main_loop(R - horizon)
        near = (x[:, 1].reshape(len(x), -1).max(axis=1) > np.log1p(0.1)) | (y > 0)
        keep = near | (rng.random(len(x)) < keep_far)
        seen += len(x)
        pos += int(y.sum())
        xs.append(x[keep].astype(np.float16))
        ys.append(y[keep])
    return (np.concatenate(xs), np.concatenate(ys),
            {"samples": seen, "positives": pos, "kept": int(sum(len(a) for a in ys))})


def train_net(net: "Net", x, y, epochs: int = 4, batch: int = 512, lr: float = 2e-3,
              seed: int = 0):
    """Adam on the samples, positives weighted by the class ratio; returns
    the mean loss of each epoch."""
    rng = np.random.default_rng(seed)
    npos = max(float(y.sum()), 1.0)
    pw = float(min(max((len(y) - npos) / npos, 1.0), 50.0))
    losses = []
    for _ in range(epochs):
        order = rng.permutation(len(y))
        tot, cnt = 0.0, 0
        for i in range(0, len(order) - batch + 1, batch):
            idx = order[i:i + batch]
            tot += net.train_step(x[idx].astype(np.float32), y[idx], lr=lr, pos_weight=pw)
            cnt += 1
        losses.append(tot / max(cnt, 1))
    return losses
