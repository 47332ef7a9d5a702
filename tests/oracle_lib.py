"""ctypes binding of the CPU oracle (oracle/liborcamrlbm.so), the checker of
every parity test. Test infrastructure only."""
import ctypes as ct
import os
import subprocess

import numpy as np

from amrlbm import Params, Physics, F_ALLOC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liborcamrlbm.so")

_lib = None


def build_oracle():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = ct.CDLL(ORACLE_SO)
        vp, i32p, dp, u8p = ct.c_void_p, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_double), ct.POINTER(ct.c_uint8)
        sig = {
            "orc_create": (vp, [ct.POINTER(Params), ct.c_int]),
            "orc_destroy": (None, [vp]),
            "orc_set_threads": (None, [vp, ct.c_int]),
            "orc_last_error": (ct.c_int, [vp]),
            "orc_level_jump_count": (ct.c_int, [vp]),
            "orc_physics": (None, [vp, ct.POINTER(Physics)]),
            "orc_set_physics": (None, [vp, ct.POINTER(Physics)]),
            "orc_set_g_collision": (ct.c_int, [vp, ct.c_int]),
            "orc_init_rising_bubble": (ct.c_int, [vp]),
            "orc_init_fields": (ct.c_int, [vp]),
            "orc_step": (ct.c_int, [vp, ct.c_int]),
            "orc_phase_times": (None, [vp, ct.POINTER(ct.c_double)]),
            "orc_min_max_levels": (None, [vp]),
            "orc_set_level_range": (None, [vp, ct.c_int, ct.c_int]),
            "orc_fill_c2": (None, [vp]), "orc_fill_c": (None, [vp]), "orc_fill_hg": (None, [vp]),
            "orc_collide": (None, [vp]), "orc_stream": (None, [vp]),
            "orc_macro_h": (None, [vp]), "orc_macro_g": (None, [vp]),
            "orc_regrid": (ct.c_int, [vp, ct.c_double, ct.c_double]),
            "orc_counts": (None, [vp, i32p]),
            "orc_get_topology": (ct.c_int, [vp] + [i32p] * 8 + [u8p, i32p, i32p]),
            "orc_set_topology": (ct.c_int, [vp, ct.c_int32] + [i32p] * 8 + [u8p, ct.c_int32, i32p, ct.c_int32]),
            "orc_get_neighbours": (ct.c_int, [vp, i32p]),
            "orc_get_leaves": (ct.c_int, [vp, i32p]),
            "orc_get_block": (ct.c_int, [vp, ct.c_int] + [dp] * 6),
            "orc_set_block": (ct.c_int, [vp, ct.c_int] + [dp] * 6),
            "orc_block_error": (ct.c_int, [vp, ct.c_int, dp]),
            "orc_diag": (ct.c_int, [vp, dp]),
            "orc_collision_block": (None, [vp, ct.c_int] + [dp] * 6),
            "orc_macro_g_block": (None, [vp, ct.c_int] + [dp] * 5),
            "orc_stream_block": (None, [vp, ct.c_int, dp]),
            "orc_biquadratic_from_fine": (None, [ct.c_int] * 4 + [dp, dp]),
            "orc_biquadratic_from_coarse": (None, [ct.c_int] * 4 + [dp, dp]),
            "orc_bilinear_from_fine": (None, [ct.c_int] * 4 + [dp, dp]),
            "orc_mrt": (None, [ct.c_double, dp, dp]),
            "orc_equilibrium": (None, [vp] + [ct.c_double] * 5 + [dp, dp]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def P(a, t=ct.c_double):
    return None if a is None else a.ctypes.data_as(ct.POINTER(t))


class Oracle:
    """The CPU restatement, with the same method names as amrlbm.AmrLbm."""

    def __init__(self, params: Params, nthreads: int = 0):
        self.L = lib()
        self.params = params
        self.nx, self.ny = params.nx, params.ny
        self.s = self.L.orc_create(ct.byref(params), nthreads)
        assert self.s, "orc_create rejected the parameters"

    def close(self):
        if self.s:
            self.L.orc_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    hshape = property(lambda self: (9, self.nx + 2, self.ny + 2))
    cshape = property(lambda self: (self.nx + 4, self.ny + 4))
    pshape = property(lambda self: (self.nx, self.ny))

    def set_threads(self, n):
        self.L.orc_set_threads(self.s, n)

    PHASES = ("Macroscopic_h", "Macroscopic_g", "collision", "advection", "Ghost_C", "Ghost_C2",
              "Ghost_hg", "refine")

    def phase_times(self):
        """Seconds per phase so far, named as Main_Loop's timers
        (AMR_Rising_2D_OMP.f90:366-375)."""
        a = (ct.c_double * 8)()
        self.L.orc_phase_times(self.s, a)
        return dict(zip(self.PHASES, list(a)))

    def error(self):
        return self.L.orc_last_error(self.s)

    def level_jumps(self):
        return self.L.orc_level_jump_count(self.s)

    def physics(self):
        ph = Physics()
        self.L.orc_physics(self.s, ct.byref(ph))
        return ph

    def set_physics(self, ph):
        self.L.orc_set_physics(self.s, ct.byref(ph))

    def set_g_collision(self, model):
        assert self.L.orc_set_g_collision(self.s, model) == 0

    def initialize_rising_bubble(self):
        rc = self.L.orc_init_rising_bubble(self.s)
        assert rc == 0, rc

    def initialize_fields(self):
        assert self.L.orc_init_fields(self.s) == 0

    def main_loop(self, n):
        rc = self.L.orc_step(self.s, n)
        assert rc == 0, rc

    def determine_min_max_levels(self):
        self.L.orc_min_max_levels(self.s)
        c = self.counts()
        return c["level_min"], c["level_max"]

    def set_level_range(self, a, b):
        self.L.orc_set_level_range(self.s, a, b)

    def fill_ghost_cells_c2(self):
        self.L.orc_fill_c2(self.s)

    def fill_ghost_cells_c(self):
        self.L.orc_fill_c(self.s)

    def fill_ghost_cells_hg(self):
        self.L.orc_fill_hg(self.s)

    def collide(self):
        self.L.orc_collide(self.s)

    def stream(self):
        self.L.orc_stream(self.s)

    def phase_field_lbm_h_g(self):
        self.collide()
        self.fill_ghost_cells_hg()
        self.stream()

    def macroscopic_values_h(self):
        self.L.orc_macro_h(self.s)

    def macroscopic_values_g(self):
        self.L.orc_macro_g(self.s)

    def refine_derefine_mesh(self, rt=None, dt=None):
        rt = self.params.refin_tol if rt is None else rt
        dt = self.params.deref_tol if dt is None else dt
        assert self.L.orc_regrid(self.s, rt, dt) == 0

    def counts(self):
        c = np.zeros(5, dtype=np.int32)
        self.L.orc_counts(self.s, P(c, ct.c_int32))
        return dict(zip(("nblks", "nleaf", "kk", "level_min", "level_max"), c.tolist()))

    def topology(self):
        n = self.counts()["nblks"]
        i32 = lambda k=1: np.zeros(n * k, dtype=np.int32)
        t = dict(level=i32(), dx=i32(), bi=i32(), bj=i32(), parent=i32(), child=i32(4),
                 nbr_owner=i32(8), nbr_slot=i32(8), flags=np.zeros(n, dtype=np.uint8))
        nfree = ct.c_int32()
        fl = np.zeros(self.params.max_blks // 4 + 1, dtype=np.int32)
        self.L.orc_get_topology(self.s, *[P(t[k], ct.c_int32) for k in
                                          ("level", "dx", "bi", "bj", "parent", "child", "nbr_owner", "nbr_slot")],
                                P(t["flags"], ct.c_uint8), ct.byref(nfree), P(fl, ct.c_int32))
        t["free_list"] = fl[: nfree.value].copy()
        t["child"] = t["child"].reshape(n, 4)
        t["nbr_owner"] = t["nbr_owner"].reshape(n, 8)
        t["nbr_slot"] = t["nbr_slot"].reshape(n, 8)
        return t

    def set_topology(self, t, kk):
        n = len(t["level"])
        c = lambda a: np.ascontiguousarray(a, dtype=np.int32).ravel()
        arrs = [c(t[k]) for k in ("level", "dx", "bi", "bj", "parent", "child", "nbr_owner", "nbr_slot")]
        fl = c(t["free_list"]) if len(t["free_list"]) else np.zeros(1, np.int32)
        rc = self.L.orc_set_topology(self.s, n, *[P(a, ct.c_int32) for a in arrs],
                                     P(np.ascontiguousarray(t["flags"], np.uint8), ct.c_uint8),
                                     len(t["free_list"]), P(fl, ct.c_int32), kk)
        assert rc == 0

    def neighbours(self):
        n = self.counts()["nblks"]
        a = np.zeros(8 * n, dtype=np.int32)
        self.L.orc_get_neighbours(self.s, P(a, ct.c_int32))
        return a.reshape(n, 8)

    def leaves(self):
        n = self.counts()["nleaf"]
        a = np.zeros(max(n, 1), dtype=np.int32)
        self.L.orc_get_leaves(self.s, P(a, ct.c_int32))
        return a[:n]

    def download_block(self, bid):
        h = np.zeros(self.hshape, order="F")
        g = np.zeros(self.hshape, order="F")
        C = np.zeros(self.cshape, order="F")
        Pp = np.zeros(self.pshape, order="F")
        Ux = np.zeros(self.pshape, order="F")
        Uy = np.zeros(self.pshape, order="F")
        rc = self.L.orc_get_block(self.s, bid, *[P(a) for a in (h, g, C, Pp, Ux, Uy)])
        assert rc == 0, (bid, rc)
        return dict(h=h, g=g, C=C, P=Pp, Ux=Ux, Uy=Uy)

    def upload_block(self, bid, h=None, g=None, C=None, P_=None, Ux=None, Uy=None):
        f = lambda a: None if a is None else np.asfortranarray(a, dtype=np.float64)
        assert self.L.orc_set_block(self.s, bid, *[P(f(a)) for a in (h, g, C, P_, Ux, Uy)]) == 0

    def block_error(self, bid):
        e = ct.c_double()
        assert self.L.orc_block_error(self.s, bid, ct.byref(e)) == 0
        return e.value

    def output(self):
        out = np.zeros(8)
        rc = self.L.orc_diag(self.s, P(out))
        d = dict(zip(("mass", "rho_min", "rho_max", "u_max", "bubble_volume",
                      "y_centroid", "rise_velocity", "phase_volume"), out.tolist()))
        d["status"] = rc
        return d

    def allocated_blocks(self):
        t = self.topology()
        return [i + 1 for i in range(len(t["level"])) if t["flags"][i] & F_ALLOC]
