"""CPU restatement of exchange_messages_sphere for a single-process sphere of
blocks (test infrastructure only: the checker of gitm_hz_exchange).

Follows exchange_messages_sphere.f90:4-95 with the transfer of
ModSphereInterface.f90:395-513 (the fields moved, at altitudes 1..nAlts)
and srcSphereAB: the neighbours of AB_SPH_module.f90:180-370 (block i =
iLat * num_long + iLong; across a connected pole the block num_long / 2
away, the corner blocks num_long / 2 +- 1 away) and the ghost-ring packing
of AB_XFER_array_util.f90 (two cells; across a pole the rows in reverse
order, the columns as they are).  Written per block and ghost region as the
library does, not through the global-index rule the CUDA kernel uses, so
the two are independent.  Arrays are the HzBlocks layout of
gitm_b200/horizontal.py: (nBlocks[, k], nAlts+4, nLats+4, nLons+4).
"""
from __future__ import annotations

import numpy as np

NSPECIES = 6
NIONS = 10
GCN = 2


def _fields(A: dict, use_ion_advection: bool, non_magnetic: bool):
    """(array, field indices) moved by pack_vars_nblk, in its order."""
    out = [(A["rho"], None), (A["velocity"], range(3)), (A["vert_vel"], range(NSPECIES)),
           (A["ndensity_s"], range(NSPECIES)), (A["temperature"], None)]
    for k in ("itemperature", "etemperature"):
        if A.get(k) is not None:
            out.append((A[k], None))
    if use_ion_advection:
        out.append((A["idensity_s"], range(NIONS)))
        out.append((A["ivelocity"] if non_magnetic else A["ivelocity_par"], range(3)))
    return out


def exchange(A: dict, n_lons: int, n_lats: int, n_alts: int, nbl: int, nbt: int, north_pole: bool = True,
             south_pole: bool = True, use_ion_advection: bool = True, non_magnetic: bool = False) -> np.ndarray:
    """In place on the host arrays of A; returns the per-block status words
    (1 = Rho < 0, 64 = Temperature < 100 in the interior)."""
    nl, nt = n_lons, n_lats
    ks = slice(2, n_alts + 2)  # altitudes 1..nAlts (array index = Fortran index + 1)

    def I(i):  # array index of Fortran lon / lat index i
        return i + 1

    # neighbours (AB_SPH_module.f90:180-370): dir -> (block, across the pole)
    def nbr(bx, by, d):
        dx, dy = d
        if dy == 0:
            return ((by * nbl + (bx + dx) % nbl), False)
        if 0 <= by + dy < nbt:
            return ((by + dy) * nbl + (bx + dx) % nbl, False)
        if (dy > 0 and not north_pole) or (dy < 0 and not south_pole):
            return None
        return (by * nbl + (bx + nbl // 2 + dx) % nbl, True)

    # the cells of the sender's pack for the receiver's ghost region (d is
    # the receiver's direction): lists of (receiver lon, lat) and (sender lon, lat)
    def region(d, pole):
        dx, dy = d
        rx = {-1: [-1, 0], 0: list(range(1, nl + 1)), 1: [nl + 1, nl + 2]}[dx]
        ry = {-1: [-1, 0], 0: list(range(1, nt + 1)), 1: [nt + 1, nt + 2]}[dy]
        # the receiver's east ghosts take the sender's first columns, its
        # west ghosts the last ones, across a pole too (the sender there
        # packs its north-west region for the receiver's north-east, ...)
        sx = {-1: [nl - 1, nl], 0: list(range(1, nl + 1)), 1: [1, 2]}[dx]
        if pole:
            # the sender packs its own north (south) rows, in reverse order
            sy = [nt, nt - 1] if dy > 0 else [2, 1]
        else:
            sy = {-1: [nt - 1, nt], 0: list(range(1, nt + 1)), 1: [1, 2]}[dy]
        return rx, ry, sx, sy

    fields = _fields(A, use_ion_advection, non_magnetic)
    dirs = [(0, 1), (0, -1), (1, 0), (-1, 0), (1, 1), (-1, 1), (1, -1), (-1, -1)]
    # the sources are interior cells, which the exchange does not write
    for by in range(nbt):
        for bx in range(nbl):
            b = by * nbl + bx
            for d in dirs:
                nb = nbr(bx, by, d)
                if nb is None:
                    continue
                sb, pole = nb
                rx, ry, sx, sy = region(d, pole)
                for arr, idx in fields:
                    for jr, js in zip(ry, sy):
                        for ir, is_ in zip(rx, sx):
                            if idx is None:
                                arr[b, ks, I(jr), I(ir)] = arr[sb, ks, I(js), I(is_)]
                            else:
                                for f in idx:
                                    arr[b, f, ks, I(jr), I(ir)] = arr[sb, f, ks, I(js), I(is_)]
    # exchange_messages_sphere.f90:35-76
    vi = A["ivelocity"] if non_magnetic else A["ivelocity_par"]
    lat = A["latitude"]
    st = np.zeros(nbl * nbt, dtype=np.uint32)
    for b in range(nbl * nbt):
        if lat[b, I(0)] < -np.pi / 2.0:
            for a in (A["velocity"], vi):
                a[b, 0:2, :, I(-1):I(0) + 1, :] = -a[b, 0:2, :, I(-1):I(0) + 1, :]
        if lat[b, I(nt + 1)] > np.pi / 2.0:
            for a in (A["velocity"], vi):
                a[b, 0:2, :, I(nt + 1):I(nt + 2) + 1, :] = -a[b, 0:2, :, I(nt + 1):I(nt + 2) + 1, :]
        # :78-88
        if A["temperature"][b, ks, 2:nt + 2, 2:nl + 2].min() < 100.0:
            st[b] |= 64
        if A["rho"][b, ks, 2:nt + 2, 2:nl + 2].min() < 0.0:
            st[b] |= 1
    return st
