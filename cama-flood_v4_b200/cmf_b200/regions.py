"""Basin-region decomposition for running one domain on several GPUs.

Mirrors the reference's MPI design (src/cmf_ctrl_maps_mod.F90:308-397, etc/options_HPC/README.md):
regions are unions of whole river basins, basins joined by a bifurcation channel go to the same
region, so no cell ever reads another region's state.  The only per-step exchange is the MIN
all-reduce of the CFL time step (CMF_MPI_ADPSTP, src/cmf_ctrl_mpi_mod.F90:261-281).

Because CALC_1D_SEQ orders cells generation by generation in row-major scan order, a region's
own sequence keeps the relative order of its cells, so every upstream sum is taken in the same
order as in the whole-domain run and the regional run is bit-identical to it.
"""
from __future__ import annotations

import os
import shutil

import numpy as np

IMIS = -9999


def _find(parent, a):
    while parent[a] != a:
        parent[a] = parent[parent[a]]
        a = parent[a]
    return a


def basin_ids(nextx: np.ndarray, nexty: np.ndarray) -> np.ndarray:
    """Flat index of the mouth each land cell drains to (-1 for ocean)."""
    ny, nx = nextx.shape
    nxf = nextx.ravel()
    nyf = nexty.ravel()
    out = np.full(nx * ny, -1, dtype=np.int64)
    for c in range(nx * ny):
        if nxf[c] == IMIS or out[c] >= 0:
            continue
        path = []
        k = c
        while True:
            if out[k] >= 0:
                root = out[k]
                break
            path.append(k)
            if nxf[k] <= 0:          # mouth (negative code)
                root = k
                break
            k = (nyf[k] - 1) * nx + (nxf[k] - 1)
        for p in path:
            out[p] = root
    return out


def region_map(nextx: np.ndarray, nexty: np.ndarray, bif_pairs, nregions: int) -> np.ndarray:
    """Region id (1..nregions) per grid cell, IMIS for ocean: bifurcation-merged basins packed
    greedily, largest first, into the currently smallest region (balance by cell count)."""
    ny, nx = nextx.shape
    b = basin_ids(nextx, nexty)
    land = np.nonzero(b >= 0)[0]
    roots = np.unique(b[land])
    parent = {int(r): int(r) for r in roots}
    for (ix, iy, jx, jy) in bif_pairs:
        a = b[(iy - 1) * nx + (ix - 1)]
        c = b[(jy - 1) * nx + (jx - 1)]
        if a >= 0 and c >= 0:
            ra, rc = _find(parent, int(a)), _find(parent, int(c))
            if ra != rc:
                parent[ra] = rc
    group = np.array([_find(parent, int(r)) for r in b[land]])
    gids, counts = np.unique(group, return_counts=True)
    order = np.argsort(-counts, kind="stable")
    load = np.zeros(nregions, dtype=np.int64)
    assign = {}
    for k in order:
        r = int(np.argmin(load))
        assign[int(gids[k])] = r + 1
        load[r] += counts[k]
    reg = np.full(nx * ny, IMIS, dtype=np.int32)
    reg[land] = np.array([assign[int(g)] for g in group], dtype=np.int32)
    return reg.reshape(ny, nx)


def read_bif_pairs(casedir: str):
    p = os.path.join(casedir, "bifprm.txt")
    if not os.path.exists(p):
        return []
    with open(p) as f:
        f.readline()
        return [tuple(int(v) for v in ln.split()[:4]) for ln in f if ln.strip()]


def split_case(casedir: str, nregions: int, outdir: str) -> list:
    """Writes one case directory per region: cells of other regions become ocean (IMIS) in nextxy,
    which is what CALC_REGION/CALC_1D_SEQ do with the reference's mpireg map.  Also writes the
    region map as mpireg.bin (int32 NX*NY, the reference's format) into casedir's copy."""
    with open(os.path.join(casedir, "diminfo.txt")) as f:
        nx = int(f.readline().split()[0])
        ny = int(f.readline().split()[0])
    raw = np.fromfile(os.path.join(casedir, "nextxy.bin"), dtype="<i4").reshape(2, ny, nx)
    reg = region_map(raw[0], raw[1], read_bif_pairs(casedir), nregions)
    dirs = []
    for r in range(1, nregions + 1):
        d = os.path.join(outdir, f"region{r}")
        if os.path.exists(d):
            shutil.rmtree(d)
        shutil.copytree(casedir, d)
        sub = raw.copy()
        outside = reg != r
        sub[0][outside] = IMIS
        sub[1][outside] = IMIS
        sub.astype("<i4").tofile(os.path.join(d, "nextxy.bin"))
        reg.astype("<i4").tofile(os.path.join(d, "mpireg.bin"))
        dirs.append(d)
    return dirs


def members_for_rank(nmembers: int, world: int, rank: int) -> list:
    """Ensemble members owned by `rank` (contiguous blocks, sizes differ by at most one)."""
    base, extra = divmod(nmembers, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def expected_nt(nxtdst: np.ndarray, rivhgt: np.ndarray, nseqriv: int, dt: float = 3600.0,
                fill: float = 0.5, pcadp: float = 0.7, pdstmth: float = 10000.0, pgrv: float = 9.8) -> int:
    """Sub-steps per outer step that CALC_ADPSTP (src/cmf_ctrl_physics_mod.F90:161-206) gives when
    every channel holds `fill` of its bank height: DT_MIN over the cells' CFL keys
    PCADP*DDST*(PGRV*DDPH)**(-0.5) (mouths use PDSTMTH), then NT = INT(DT/DT_MIN - 0.01) + 1.  An
    estimate of a member's work per outer step before the run has a state of its own."""
    n = nxtdst.size
    ddst = np.where(np.arange(n) < nseqriv, nxtdst, pdstmth)
    ddph = np.maximum(rivhgt * fill, 0.01)
    dt_min = min(dt, float(np.min((pcadp * ddst) * (pgrv * ddph) ** -0.5))) if n else dt
    return int(dt * (1.0 / dt_min) - float(np.float32(0.01))) + 1


def pack_units(loads, nmembers: int, world: int) -> list:
    """Members x domains over `world` ranks: unit (d, m) is member m of domain d, with weight
    loads[d] (cells x expected NT of one member).  Greedy bin-packing, largest unit first (ties:
    lower domain, then lower member), each unit to the rank with the least load so far (ties: lower
    rank).  Returns, per rank, a list over domains of the member ids it owns (ascending); every unit
    is owned once, and no rank's load exceeds the mean by more than the largest unit."""
    loads = [float(x) for x in loads]
    order = sorted(((d, m) for d in range(len(loads)) for m in range(nmembers)),
                   key=lambda u: (-loads[u[0]], u[0], u[1]))
    acc = [0.0] * world
    owned = [[[] for _ in loads] for _ in range(world)]
    for d, m in order:
        r = min(range(world), key=lambda k: (acc[k], k))
        acc[r] += loads[d]
        owned[r][d].append(m)
    for per in owned:
        for ms in per:
            ms.sort()
    return owned
