"""Helpers that compare the B200 pool (amrlbm.AmrLbm) with the CPU oracle.

Integer state (topology, flags, neighbour pointers and values, leaf list,
free list, counters) must be identical. FP64 fields must be identical too:
the device path evaluates every formula in the reference's order with no
FMA contraction, so its results equal the oracle's IEEE double evaluation;
``==`` is used, so +0 and -0 compare equal.
"""
import numpy as np

from amrlbm import F_ALLOC, F_LEAF


def compare_counts(gpu, orc):
    g, o = gpu.counts(), orc.counts()
    assert g == o, f"counts differ: gpu {g} oracle {o}"


def compare_topology(gpu, orc, check_flags=True):
    tg, to = gpu.topology(), orc.topology()
    for k in ("level", "dx", "bi", "bj", "parent", "child", "nbr_owner", "nbr_slot",
              "free_list"):
        a, b = tg[k], to[k]
        assert a.shape == b.shape and np.array_equal(a, b), f"topology '{k}' differs at " \
            f"{np.argwhere(a != b)[:8].tolist() if a.shape == b.shape else (a.shape, b.shape)}"
    if check_flags:
        diff = np.nonzero(tg["flags"] != to["flags"])[0]
        assert diff.size == 0, f"flags differ at ids {(diff + 1)[:8].tolist()}: " \
            f"gpu {tg['flags'][diff[:8]].tolist()} oracle {to['flags'][diff[:8]].tolist()}"
    assert np.array_equal(gpu.leaves(), orc.leaves()), "leaf lists differ"
    assert np.array_equal(gpu.neighbours(), orc.neighbours()), "resolved neighbours differ"
    return to


def field_ids(orc, leaves_only=False):
    t = orc.topology()
    ids = [i + 1 for i in range(len(t["level"]))
           if t["flags"][i] & (F_LEAF if leaves_only else F_ALLOC)]
    return np.array(ids, dtype=np.int32)


def _first_diff(a, b):
    bad = np.argwhere(~((a == b) | (np.isnan(a) & np.isnan(b))))
    return bad[:5].tolist()


def compare_fields(gpu, orc, ids=None, fields=("h", "g", "C", "P", "Ux", "Uy"),
                   h_interior_only=False, c_rings=2, rtol=0.0):
    """Fields of `ids` (default: every allocated block). c_rings: how many C
    ghost rings to compare (0, 1, 2). rtol 0 means exact."""
    if ids is None:
        ids = field_ids(orc)
    nx, ny = orc.nx, orc.ny
    g = gpu.download_fields(ids)
    for i, bid in enumerate(ids):
        o = orc.download_block(int(bid))
        for k in fields:
            a = g[k][i].reshape(o[k].shape, order="F")
            b = o[k]
            if k in ("h", "g") and h_interior_only:
                a, b = a[:, 1:nx + 1, 1:ny + 1], b[:, 1:nx + 1, 1:ny + 1]
            if k == "C" and c_rings < 2:
                r = 2 - c_rings
                a, b = a[r:nx + 4 - r, r:ny + 4 - r], b[r:nx + 4 - r, r:ny + 4 - r]
            if rtol == 0.0:
                ok = np.array_equal(a, b)
            else:
                ok = np.allclose(a, b, rtol=rtol, atol=rtol * max(1.0, np.abs(b).max()))
            assert ok, f"block {bid} field {k} differs at {_first_diff(a, b)}: " \
                f"max |diff| {np.nanmax(np.abs(a - b)):.3e}"


def compare_state(gpu, orc, **kw):
    compare_counts(gpu, orc)
    compare_topology(gpu, orc)
    compare_fields(gpu, orc, **kw)


def copy_state_to_gpu(orc, gpu):
    """Loads the oracle's complete state (topology, free list, fields) into the pool."""
    t = orc.topology()
    c = orc.counts()
    gpu.set_topology(t, c["kk"])
    gpu.set_level_range(c["level_min"], c["level_max"])
    ids = field_ids(orc)
    fields = {k: [] for k in ("h", "g", "C", "P", "Ux", "Uy")}
    for bid in ids:
        o = orc.download_block(int(bid))
        for k in fields:
            fields[k].append(np.asfortranarray(o[k]).ravel(order="F"))
    gpu.upload_fields(ids, {k: np.concatenate(v) for k, v in fields.items()})


def randomize_leaves(orc, seed, c_lo=-0.1, c_hi=1.1):
    """Random fields on every leaf of the oracle (C including both rings)."""
    rng = np.random.default_rng(seed)
    for bid in field_ids(orc, leaves_only=True):
        b = orc.download_block(int(bid))
        C = rng.uniform(c_lo, c_hi, size=b["C"].shape)
        P = rng.uniform(-1e-3, 1e-3, size=b["P"].shape)
        Ux = rng.uniform(-0.02, 0.02, size=b["Ux"].shape)
        Uy = rng.uniform(-0.02, 0.02, size=b["Uy"].shape)
        w = np.array([16, 4, 4, 4, 4, 1, 1, 1, 1]) / 36.0
        h = w[:, None, None] * rng.uniform(0.0, 1.0, size=b["h"].shape)
        g = w[:, None, None] * rng.uniform(-1e-3, 1e-3, size=b["g"].shape)
        orc.upload_block(int(bid), h, g, C, P, Ux, Uy)


def assert_physical(d, u_bound, label=""):
    """The Output diagnostics of a physical rising-bubble state
    (AMR_Rising_2D_OMP.f90:456-489): every leaf value finite, the velocity far
    below the lattice sound speed 1/sqrt(3), the light phase's density
    positive, the bubble rising."""
    assert d.get("status", 0) == 0, f"{label}: non-finite values"
    for k in ("mass", "rho_min", "rho_max", "u_max", "y_centroid", "rise_velocity"):
        assert np.isfinite(d[k]), f"{label}: {k} = {d[k]}"
    assert d["u_max"] < u_bound, f"{label}: u_max {d['u_max']} >= {u_bound}"
    assert d["rho_min"] > 0.0, f"{label}: rho_min {d['rho_min']}"
    assert d["rise_velocity"] > 0.0, f"{label}: rise velocity {d['rise_velocity']}"
