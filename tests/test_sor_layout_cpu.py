"""Host check of the SOR lane layouts the library builds (no GPU).

gpg_sor_layout() reports the constants of every (precision, ghost size,
layout); this test restates the kernel's lane decode (sor_solve_patch in
csrc/sor_kernel.cuh) and checks, for every layout that is built:

  * the shared-cube address map (colour, z, y, x-slot) is one-to-one and stays
    inside the team's 2 * N * PP elements;
  * the active lanes update every interior cell exactly once per sweep;
  * every neighbour a pass reads -- from shared memory or from the lane's own
    registers -- is the cell the 7-point stencil names, and the reload plane
    of a split column is inside the cube;
and that the one-row layout and the two-row default of FP64 ghost 5 need the
shared-memory wavefronts per patch-sweep the layout search reported (1024, and
768 in the passes + 32 reloads across the split = 800; a 64-bit access costs,
per half-warp, the largest number of distinct words one bank holds).
"""
import ctypes as C

import pytest

from gpg.lib import check, library

FIELDS = ("Z", "Y", "MH", "R", "P", "PADZ", "U", "BLOCK", "TEAM", "PP", "FITS")


def layout(rs, g, variant):
    f = (C.c_int * len(FIELDS))()
    check(library().gpg_sor_layout(rs, g, variant, f))
    return dict(zip(FIELDS, f))


def layouts():
    seen = {}
    for rs in (4, 8):
        for g in range(1, 6):
            for v in range(library().gpg_sor_variant_count()):
                L = layout(rs, g, v)
                if L["FITS"]:
                    seen.setdefault((rs, g, L["Z"], L["Y"]), v)
    return sorted(seen.items())


def addr(L, n, x, y, z):
    return (((x + y + z + 1) & 1) * n + z) * L["PP"] + y * L["P"] + ((x + 1) >> 1)


def lanes(L, g):
    """Active lanes as (y, h, zbase) -- the kernel's decode."""
    m = 6 + 2 * g
    half = m // 2
    nblock = (2 if L["Y"] == 1 else 1) * L["Z"]
    out = []
    for tid in range(L["TEAM"]):
        blk, li = divmod(tid, L["BLOCK"])
        r, h0 = divmod(li, L["R"])
        if not (blk < nblock and r < m // 2 and h0 < half):
            continue
        cls = blk // L["Z"] if L["Y"] == 1 else 0
        y = 2 * r + 1 + cls
        zbase = (blk - cls * L["Z"]) * L["MH"]
        out.append((tid, y, h0, zbase))
    return out


@pytest.mark.parametrize("key,variant", layouts(), ids=lambda k: str(k))
def test_layout_indexing(key, variant):
    rs, g, _, _ = key
    L = layout(rs, g, variant)
    n, m = 8 + 2 * g, 6 + 2 * g
    cube = 2 * n * L["PP"]
    seen = set()
    for z in range(n):
        for y in range(n):
            for x in range(n):
                a = addr(L, n, x, y, z)
                assert 0 <= a < cube and a not in seen
                seen.add(a)
    updated = set()
    for tid, y, h, zbase in lanes(L, g):
        own = y * L["P"] + h + 1
        for p in (0, 1):
            oc = 1 - p
            for zz in range(1, L["MH"] + 1):
                z = zbase + zz
                for r in range(L["Y"]):
                    yr = y + r
                    x = 2 * h + 1 if ((yr + z + p) & 1) == 0 else 2 * h + 2
                    cell = (x, yr, z)
                    assert cell not in updated
                    updated.add(cell)
                    slot = own + r * L["P"]
                    assert addr(L, n, x, yr, z) == (p * n + z) * L["PP"] + slot
                    # every stencil neighbour: in-lane registers hold the same
                    # pair's slots of the lane's rows at heights zbase..zbase+MH+1
                    for (xn, yn, zn) in ((x + 1, yr, z), (x - 1, yr, z), (x, yr + 1, z), (x, yr - 1, z),
                                         (x, yr, z + 1), (x, yr, z - 1)):
                        a = addr(L, n, xn, yn, zn)
                        assert 0 <= a < cube
                        assert (((xn + yn + zn + 1) & 1) == oc)  # the other colour
                        in_lane = (yn in range(y, y + L["Y"]) and (xn + 1) >> 1 == h + 1
                                   and zbase <= zn <= zbase + L["MH"] + 1)
                        if not in_lane:
                            # shared memory: the outside x slot or the row outside the lane's rows
                            assert (yn == yr and abs((xn + 1) // 2 - (h + 1)) == 1) or yn in (y - 1, y + L["Y"])
            if L["Z"] == 2:
                bz = zbase + (0 if zbase else L["MH"] + 1)
                assert 0 <= bz < n
    assert len(updated) == m ** 3


def wavefronts_per_sweep(L, g, f64=True):
    """Shared-memory wavefronts of one sweep (loads and stores of both passes)."""
    group, banks = (16, 16) if f64 else (32, 32)
    act = {tid: (y, h, zb) for tid, y, h, zb in lanes(L, g)}
    total = 0
    for p in (0, 1):
        for zz in range(1, L["MH"] + 1):
            kinds = []
            for r in range(L["Y"]):
                kinds += [("x", r), ("st", r)]
                if r == 0:
                    kinds.append(("ym", r))
                if r == L["Y"] - 1:
                    kinds.append(("yp", r))
            for kind, r in kinds:
                for g0 in range(0, L["TEAM"], group):
                    words = {}
                    for tid in range(g0, g0 + group):
                        if tid not in act:
                            continue
                        y, h, zb = act[tid]
                        yr, z = y + r, zb + zz
                        own = zb * L["PP"] + yr * L["P"] + h + 1
                        left = ((yr + z + p) & 1) == 0
                        a = {"x": own - 1 if left else own + 1, "st": own, "ym": own - L["P"],
                             "yp": own + L["P"]}[kind]
                        words.setdefault(a % banks, set()).add(a)
                    if words:
                        total += max(len(s) for s in words.values())
    return total


def test_wavefronts_of_fp64_g5_layouts():
    assert wavefronts_per_sweep(layout(8, 5, 0), 5) == 1024   # one row, whole column
    # two rows, half columns: 768 in the passes + 32 reloads across the split
    assert wavefronts_per_sweep(layout(8, 5, 11), 5) == 768
