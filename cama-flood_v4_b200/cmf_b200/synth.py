"""Seeded synthetic CaMa-Flood cases written in the reference's own file formats.

Every file this module writes is the format the Fortran model reads, so a Fortran build of
the model could run the same case:

* ``diminfo.txt``      -- read by CMF_CONFIG_NMLIST (src/cmf_ctrl_nmlist_mod.F90:197-212)
* ``nextxy.bin``       -- 2 int32 NX*NY records, IX fastest (src/cmf_ctrl_maps_mod.F90:238-242);
                          river mouth code -9, ocean IMIS=-9999
* ``ctmare/elevtn/nxtdst/rivlen/rivwth/rivhgt/rivman.bin`` -- float32 NX*NY maps
                          (READ_TOPO_BIN, src/cmf_ctrl_maps_mod.F90:745-849)
* ``fldhgt.bin``       -- NLFP float32 records (src/cmf_ctrl_maps_mod.F90:789-797)
* ``bifprm.txt``       -- ``NPTHOUT NPTHLEV`` then ``IX IY JX JY DST ELV DPH WTH(1:NPTHLEV)``
                          (READ_BIFPARAM, src/cmf_ctrl_maps_mod.F90:548,564)
* ``levhgt.bin/levfrc.bin`` -- float32 levee maps (CMF_LEVEE_INIT, src/cmf_ctrl_levee_mod.F90:124-133)
* ``dam_params.csv``   -- NDAM, header, one row per dam (CMF_DAMOUT_INIT,
                          src/cmf_ctrl_damout_mod.F90:141-179)
* ``input_cmf.nam``    -- the namelist groups the physics reads (NRUNVER, NDIMTIME, NPARAM, NMAP,
                          NLEVEE, NDAMOUT)

The geometry laws are: upstream area A [km2] is the flow accumulation of ``ctmare``;
``rivwth = 5 A^0.5`` m; ``rivhgt = 0.3 A^0.4`` m; ``rivlen ~ LogNormal(median 15 km, sigma 0.5)``;
``nxtdst = rivlen``; ``ctmare = 2.25e8 m2 * LogNormal(0, 0.2)``; outlet ``elevtn = 0`` and going
upstream ``elevtn(i) = elevtn(next) + S_i * nxtdst(i)`` with ``S_i ~ U(1e-5, 1e-3)``; ``fldhgt`` is the
cumulative sum of 10 positive ``U(0, 2 m)`` increments; ``rivman = 0.03``.
"""
from __future__ import annotations

import heapq
import os
from dataclasses import dataclass, field

import numpy as np

IMIS = -9999
MOUTH_CODE = -9
NLFP = 10

_NB = [(-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]


@dataclass
class CaseSpec:
    """Options of one synthetic case (names follow the reference namelist)."""

    name: str = "cfg0"
    nx: int = 100
    ny: int = 100
    land_frac: float = 1.0          # 1.0: every grid cell is land
    n_mouths: int = 20              # used when land_frac == 1.0 (mouths on the grid edge)
    mouth_prob: float = 0.1         # coastal cells that become mouths (land_frac < 1)
    seed: int = 0
    lpthout: bool = False
    npthout: int = 0
    npthlev: int = 5
    llevee: bool = False
    levee_frac: float = 0.10
    ldamout: bool = False
    ndam: int = 0
    dt: float = 3600.0
    ifrq_inp: int = 24
    rivhgt_scale: float = 1.0       # stress variants lower the banks to force floodplain flow
    fldhgt_inc_max: float = 2.0
    extra: dict = field(default_factory=dict)


# ----------------------------------------------------------------------------------------
# network
# ----------------------------------------------------------------------------------------
def _land_mask(spec: CaseSpec, rng: np.random.Generator) -> np.ndarray:
    if spec.land_frac >= 1.0:
        return np.ones((spec.ny, spec.nx), dtype=bool)
    from scipy.ndimage import gaussian_filter

    noise = rng.standard_normal((spec.ny, spec.nx))
    sig = max(2.0, min(spec.nx, spec.ny) / 30.0)
    field_ = gaussian_filter(noise, sigma=sig, mode=("nearest", "wrap"))
    thr = np.quantile(field_, 1.0 - spec.land_frac)
    land = field_ > thr
    # keep the poles as ocean so that every basin drains to a coast
    land[0, :] = False
    land[-1, :] = False
    return land


def _mouths(spec: CaseSpec, land: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    ny, nx = land.shape
    if spec.land_frac >= 1.0:
        edge = []
        for ix in range(nx):
            edge.append((0, ix))
            edge.append((ny - 1, ix))
        for iy in range(1, ny - 1):
            edge.append((iy, 0))
            edge.append((iy, nx - 1))
        pick = rng.choice(len(edge), size=spec.n_mouths, replace=False)
        out = np.zeros_like(land)
        for p in pick:
            out[edge[p]] = True
        return out
    ocean = ~land
    coast = np.zeros_like(land)
    for dx, dy in _NB:
        sh = np.roll(np.roll(ocean, dy, axis=0), dx, axis=1)
        coast |= sh
    coast &= land
    mouths = coast & (rng.random(land.shape) < spec.mouth_prob)
    # every connected land component needs one mouth
    from scipy.ndimage import label

    lab, nlab = label(land, structure=np.ones((3, 3)))
    has = np.zeros(nlab + 1, dtype=bool)
    has[np.unique(lab[mouths])] = True
    missing = np.nonzero(~has[1:])[0] + 1
    if len(missing):
        cy, cx = np.nonzero(coast)
        cl = lab[cy, cx]
        order = rng.permutation(len(cy))
        seen = set()
        for k in order:
            c = cl[k]
            if not has[c] and c not in seen:
                seen.add(c)
                mouths[cy[k], cx[k]] = True
    return mouths


_SYNTH_LIB = None


def _native():
    """The generator's sequential loops in C++ (lib/libcmf_synth.so, built by build.py)."""
    global _SYNTH_LIB
    if _SYNTH_LIB is None:
        import ctypes as C

        pkg = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        path = os.path.join(pkg, "lib", "libcmf_synth.so")
        if not os.path.exists(path):                  # host C++ only: build it in place (g++)
            import importlib.util

            spec = importlib.util.spec_from_file_location("cmf_build", os.path.join(pkg, "build.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build_synth()
        lib = C.CDLL(path)
        P = C.c_void_p
        lib.cmf_synth_grow_forest.argtypes = [C.c_int32, C.c_int32, P, P, C.c_int64, P, C.c_int64, P, P]
        lib.cmf_synth_grow_forest.restype = C.c_int64
        lib.cmf_synth_accumulate.argtypes = [C.c_int64, P, P, P]
        lib.cmf_synth_accumulate.restype = None
        lib.cmf_synth_elevation.argtypes = [C.c_int64, P, P, P, P, P]
        lib.cmf_synth_elevation.restype = None
        _SYNTH_LIB = lib
    return _SYNTH_LIB


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _grow_forest(land: np.ndarray, mouths: np.ndarray, rng: np.random.Generator):
    """Randomised priority-first growth from the mouths over land (8-neighbour D8 tree).

    Returns (down, order): ``down`` holds the flat downstream index (-1 for mouths, -2 for
    ocean or unreached) and ``order`` lists land cells parent-first.  Native loop; the same
    search as `_grow_forest_py` (identical output)."""
    ny, nx = land.shape
    ncell = nx * ny
    landf = np.ascontiguousarray(land.ravel(), dtype=np.uint8)
    mflat = np.ascontiguousarray(np.nonzero(mouths.ravel())[0], dtype=np.int64)
    costs = rng.random(ncell * 8 + 16) + 0.05
    down = np.empty(ncell, dtype=np.int64)
    order = np.empty(ncell, dtype=np.int64)
    n = _native().cmf_synth_grow_forest(nx, ny, _ptr(landf), _ptr(mflat), mflat.size, _ptr(costs), costs.size,
                                        _ptr(down), _ptr(order))
    if n < 0:
        raise RuntimeError("cmf_synth_grow_forest: bad arguments")
    return down, order[:n].copy()


def _accumulate(order: np.ndarray, down: np.ndarray, upa: np.ndarray) -> None:
    """upa[down[c]] += upa[c] in reverse visiting order (native; as `_accumulate_py`)."""
    _native().cmf_synth_accumulate(order.size, _ptr(order), _ptr(down), _ptr(upa))


def _elevation(order: np.ndarray, down: np.ndarray, slope: np.ndarray, length: np.ndarray, elev: np.ndarray) -> None:
    """elev[c] = elev[down[c]] + slope[c] * length[c] in visiting order (native; as `_elevation_py`)."""
    _native().cmf_synth_elevation(order.size, _ptr(order), _ptr(down), _ptr(slope), _ptr(length), _ptr(elev))


def _accumulate_py(order, down, upa) -> None:
    for c in order[::-1]:
        d = down[c]
        if d >= 0:
            upa[d] += upa[c]


def _elevation_py(order, down, slope, length, elev) -> None:
    for c in order:
        d = down[c]
        if d >= 0:
            elev[c] = elev[d] + slope[c] * length[c]


def _grow_forest_py(land: np.ndarray, mouths: np.ndarray, rng: np.random.Generator):
    """Python statement of the forest growth (the check of the native loop)."""
    ny, nx = land.shape
    ncell = nx * ny
    down = np.full(ncell, -2, dtype=np.int64)
    landf = land.ravel()
    visited = np.zeros(ncell, dtype=bool)
    heap = []
    mflat = np.nonzero(mouths.ravel())[0]
    for m in mflat:
        heap.append((0.0, int(m), -1))
    heapq.heapify(heap)
    order = []
    # pre-draw random step costs in bulk
    costs = rng.random(ncell * 8 + 16) + 0.05
    ci = 0
    while heap:
        pr, c, frm = heapq.heappop(heap)
        if visited[c]:
            continue
        visited[c] = True
        down[c] = frm
        order.append(c)
        cy, cx = divmod(c, nx)
        for dx, dy in _NB:
            jx = cx + dx
            jy = cy + dy
            if jx < 0 or jx >= nx or jy < 0 or jy >= ny:
                continue
            j = jy * nx + jx
            if visited[j] or not landf[j]:
                continue
            w = costs[ci] * (1.4142 if (dx and dy) else 1.0)
            ci += 1
            if ci >= len(costs):
                ci = 0
            heapq.heappush(heap, (pr + w, j, c))
    return down, np.asarray(order, dtype=np.int64)


# ----------------------------------------------------------------------------------------
# case generation
# ----------------------------------------------------------------------------------------
@dataclass
class Case:
    spec: CaseSpec
    nx: int
    ny: int
    nextx: np.ndarray   # int32 [NY,NX], 1-based, -9 mouth, -9999 ocean
    nexty: np.ndarray
    maps: dict          # float32 [NY,NX] maps
    fldhgt: np.ndarray  # float32 [NLFP,NY,NX]
    order: np.ndarray   # parent-first flat land indices
    uparea: np.ndarray  # float64 [NY*NX] km2
    bif_rows: list = field(default_factory=list)
    levee: dict = field(default_factory=dict)
    dams: list = field(default_factory=list)


def make_case(spec: CaseSpec) -> Case:
    rng = np.random.default_rng(spec.seed)
    land = _land_mask(spec, rng)
    mouths = _mouths(spec, land, rng)
    down, order = _grow_forest(land, mouths, rng)
    ny, nx = land.shape
    ncell = nx * ny
    reached = down > -2
    nextx = np.full(ncell, IMIS, dtype=np.int32)
    nexty = np.full(ncell, IMIS, dtype=np.int32)
    ism = reached & (down == -1)
    isr = reached & (down >= 0)
    nextx[ism] = MOUTH_CODE
    nexty[ism] = MOUTH_CODE
    dwn = down[isr]
    nextx[isr] = (dwn % nx + 1).astype(np.int32)
    nexty[isr] = (dwn // nx + 1).astype(np.int32)

    # geometry laws
    ctmare = np.zeros(ncell)
    ctmare[reached] = 2.25e8 * rng.lognormal(0.0, 0.2, size=int(reached.sum()))
    ctm32 = ctmare.astype(np.float32).astype(np.float64)
    upa = ctm32.copy()
    _accumulate(order, down, upa)
    upa_km2 = upa * 1e-6
    rivlen = np.zeros(ncell)
    rivlen[reached] = 15000.0 * rng.lognormal(0.0, 0.5, size=int(reached.sum()))
    rivlen32 = rivlen.astype(np.float32).astype(np.float64)
    slope = rng.uniform(1e-5, 1e-3, size=ncell)
    elev = np.zeros(ncell)
    _elevation(order, down, slope, rivlen32, elev)
    rivwth = np.where(reached, 5.0 * np.sqrt(upa_km2), 0.0)
    rivhgt = np.where(reached, 0.3 * np.power(np.maximum(upa_km2, 1e-12), 0.4) * spec.rivhgt_scale, 0.0)
    rivman = np.where(reached, 0.03, 0.0)
    incs = rng.uniform(0.0, spec.fldhgt_inc_max, size=(NLFP, ncell))
    incs = np.maximum(incs, 1e-3)
    fld = np.cumsum(incs, axis=0)
    fld[:, ~reached] = 0.0

    def m32(a):
        out = np.where(reached, a, -9999.0).astype(np.float32)
        return out.reshape(ny, nx)

    maps = {
        "ctmare": m32(ctmare),
        "elevtn": m32(elev),
        "nxtdst": m32(rivlen32),
        "rivlen": m32(rivlen32),
        "rivwth": m32(rivwth),
        "rivhgt": m32(rivhgt),
        "rivman": m32(rivman),
    }
    fldhgt = np.where(reached[None, :], fld, -9999.0).astype(np.float32).reshape(NLFP, ny, nx)
    case = Case(spec, nx, ny, nextx.reshape(ny, nx), nexty.reshape(ny, nx), maps, fldhgt, order, upa_km2)

    land_idx = np.nonzero(reached)[0]
    if spec.lpthout and spec.npthout > 0:
        case.bif_rows = _make_bifurcations(spec, rng, land_idx, down, nx, ny, reached, maps)
    if spec.llevee:
        lh = np.zeros(ncell, dtype=np.float32)
        lf = np.ones(ncell, dtype=np.float32)
        sel = land_idx[rng.random(len(land_idx)) < spec.levee_frac]
        lh[sel] = rng.uniform(1.0, 5.0, size=len(sel))
        lf[sel] = rng.uniform(0.1, 0.9, size=len(sel))
        lh[~reached] = -9999.0
        lf[~reached] = -9999.0
        case.levee = {"levhgt": lh.reshape(ny, nx), "levfrc": lf.reshape(ny, nx)}
    if spec.ldamout and spec.ndam > 0:
        case.dams = _make_dams(spec, rng, land_idx, down, nx, upa_km2)
    return case


def _make_bifurcations(spec, rng, land_idx, down, nx, ny, reached, maps):
    rows = []
    elev = maps["elevtn"].ravel().astype(np.float64)
    hgt = maps["rivhgt"].ravel().astype(np.float64)
    wth = maps["rivwth"].ravel().astype(np.float64)
    tries = 0
    used = set()
    while len(rows) < spec.npthout and tries < spec.npthout * 50:
        tries += 1
        c = int(land_idx[rng.integers(len(land_idx))])
        cy, cx = divmod(c, nx)
        dx, dy = _NB[rng.integers(8)]
        jx, jy = cx + dx, cy + dy
        if jx < 0 or jx >= nx or jy < 0 or jy >= ny:
            continue
        j = jy * nx + jx
        if not reached[j] or down[c] == j or down[j] == c or (c, j) in used:
            continue
        used.add((c, j))
        dst = float(rng.uniform(5000.0, 30000.0))
        pelv = float(elev[c])
        pdph = float(0.5 * hgt[c])
        wths = [float(0.3 * wth[c])]
        for _ in range(spec.npthlev - 1):
            wths.append(0.0 if rng.random() < 0.3 else float(rng.uniform(50.0, 500.0)))
        rows.append((cx + 1, cy + 1, jx + 1, jy + 1, dst, pelv, pdph, wths))
    return rows


def _make_dams(spec, rng, land_idx, down, nx, upa_km2):
    big = land_idx[(down[land_idx] >= 0)]
    big = big[np.argsort(-upa_km2[big])]
    pool = big[: max(spec.ndam * 5, spec.ndam)]
    pick = rng.choice(len(pool), size=min(spec.ndam, len(pool)), replace=False)
    dams = []
    for k, p in enumerate(pick):
        c = int(pool[p])
        cy, cx = divmod(c, nx)
        tot_mcm = float(1e8 * rng.lognormal(0.0, 1.0) * 1e-6)
        ffrac = float(rng.uniform(0.2, 0.5))
        fld_mcm = tot_mcm * ffrac
        con_mcm = tot_mcm - fld_mcm
        qn = float(2.0e-3 * upa_km2[c] * 1e6 / 86400.0)
        qf = 3.0 * qn
        dams.append((k + 1, f"DAM{k + 1:05d}", 0.0, 0.0, float(upa_km2[c]), cx + 1, cy + 1,
                     fld_mcm, con_mcm, tot_mcm, qn, qf))
    return dams


# ----------------------------------------------------------------------------------------
# writers (reference formats)
# ----------------------------------------------------------------------------------------
def write_case(case: Case, outdir: str) -> str:
    os.makedirs(outdir, exist_ok=True)
    s = case.spec
    with open(os.path.join(outdir, "diminfo.txt"), "w") as f:
        f.write(f"{case.nx:>12d}     !! nXX\n{case.ny:>12d}     !! nYY\n{NLFP:>12d}     !! floodplain layer\n")
        f.write(f"{case.nx:>12d}     !! input nXX\n{case.ny:>12d}     !! input nYY\n{1:>12d}     !! input num\n")
        f.write("none\n")
        f.write(f"{-180.0:12.3f}     !! west  edge\n{180.0:12.3f}     !! east  edge\n")
        f.write(f"{90.0:12.3f}     !! north edge\n{-90.0:12.3f}     !! south edge\n")
    with open(os.path.join(outdir, "nextxy.bin"), "wb") as f:
        f.write(case.nextx.astype("<i4").tobytes())
        f.write(case.nexty.astype("<i4").tobytes())
    for k, v in case.maps.items():
        v.astype("<f4").tofile(os.path.join(outdir, f"{k}.bin"))
    case.fldhgt.astype("<f4").tofile(os.path.join(outdir, "fldhgt.bin"))
    if case.bif_rows:
        with open(os.path.join(outdir, "bifprm.txt"), "w") as f:
            f.write(f"{len(case.bif_rows):8d}{s.npthlev:8d}   npthout, npthlev, IX,IY,JX,JY,length,elevtn,depth,width\n")
            for (ix, iy, jx, jy, dst, pelv, pdph, wths) in case.bif_rows:
                w = " ".join(f"{x:.6f}" for x in wths)
                f.write(f"{ix:8d}{iy:8d}{jx:8d}{jy:8d} {dst:.6f} {pelv:.6f} {pdph:.6f} {w}\n")
    if case.levee:
        case.levee["levhgt"].astype("<f4").tofile(os.path.join(outdir, "levhgt.bin"))
        case.levee["levfrc"].astype("<f4").tofile(os.path.join(outdir, "levfrc.bin"))
    if case.dams:
        with open(os.path.join(outdir, "dam_params.csv"), "w") as f:
            f.write(f"{len(case.dams)}\n")
            f.write("GRAND_ID,DamName,DamLat,DamLon,area_CaMa,DamIX,DamIY,FldVol_mcm,ConVol_mcm,TotalVol_mcm,Qn,Qf\n")
            for d in case.dams:
                f.write("%d,%s,%.4f,%.4f,%.6f,%d,%d,%.6f,%.6f,%.6f,%.6f,%.6f\n" % d)
    _write_namelist(case, outdir)
    return outdir


def _fl(b: bool) -> str:
    return ".TRUE." if b else ".FALSE."


def _write_namelist(case: Case, outdir: str) -> None:
    s = case.spec
    lines = [
        "&NRUNVER",
        "LADPSTP  = .TRUE.",
        "LFPLAIN  = .TRUE.",
        "LKINE    = .FALSE.",
        "LFLDOUT  = .TRUE.",
        f"LPTHOUT  = {_fl(s.lpthout)}",
        f"LDAMOUT  = {_fl(s.ldamout)}",
        f"LLEVEE   = {_fl(s.llevee)}",
        "LSPAMAT  = .TRUE.",
        "LRESTART = .FALSE.",
        "LOUTPUT  = .FALSE.",
        "/",
        "&NDIMTIME",
        'CDIMINFO = "diminfo.txt"',
        f"DT       = {s.dt:.1f}",
        f"IFRQ_INP = {s.ifrq_inp}",
        "/",
        "&NPARAM",
        "PMANRIV  = 0.03D0",
        "PMANFLD  = 0.10D0",
        "PGRV     = 9.8D0",
        "PDSTMTH  = 10000.D0",
        "PCADP    = 0.7",
        "/",
        "&NMAP",
        "LMAPCDF  = .FALSE.",
        'CNEXTXY  = "nextxy.bin"',
        'CGRAREA  = "ctmare.bin"',
        'CELEVTN  = "elevtn.bin"',
        'CNXTDST  = "nxtdst.bin"',
        'CRIVLEN  = "rivlen.bin"',
        'CFLDHGT  = "fldhgt.bin"',
        'CRIVWTH  = "rivwth.bin"',
        'CRIVHGT  = "rivhgt.bin"',
        'CRIVMAN  = "rivman.bin"',
        'CPTHOUT  = "bifprm.txt"',
        "/",
        "&NLEVEE",
        'CLEVHGT  = "levhgt.bin"',
        'CLEVFRC  = "levfrc.bin"',
        "/",
        "&NDAMOUT",
        'CDAMFILE = "dam_params.csv"',
        "LDAMTXT  = .FALSE.",
        "LDAMH22  = .FALSE.",
        "/",
    ]
    with open(os.path.join(outdir, "input_cmf.nam"), "w") as f:
        f.write("\n".join(lines) + "\n")


# ----------------------------------------------------------------------------------------
# forcing
# ----------------------------------------------------------------------------------------
DROFUNIT = 86400000.0  # mm/day -> m/s (src/cmf_ctrl_forcing_mod.F90, namelist NFORCE default for mm/day)


def make_inpmat(nx: int, ny: int, i1seqx: np.ndarray, i1seqy: np.ndarray, grarea: np.ndarray, factor: int = 2,
                inpn: int = 3, seed: int = 0):
    """Synthetic input matrix for runoff on a grid `factor` times coarser than the map: each cell
    draws from the coarse cell that contains it and from up to inpn - 1 neighbours, with areas that
    sum to the cell area (mass conserving); unused entries have INPX = 0.  Returns
    (nxin, nyin, inpx, inpy, inpa) in sequence order, [inpn][NSEQ]."""
    rng = np.random.default_rng(seed)
    n = i1seqx.size
    nxin, nyin = (nx + factor - 1) // factor, (ny + factor - 1) // factor
    inpx = np.zeros((inpn, n), dtype=np.int32)
    inpy = np.zeros((inpn, n), dtype=np.int32)
    inpa = np.zeros((inpn, n), dtype=np.float32)
    cx, cy = (i1seqx - 1) // factor + 1, (i1seqy - 1) // factor + 1
    w = rng.dirichlet(np.ones(inpn), size=n).T * (rng.random((inpn, n)) > 0.2)
    w[0] = np.maximum(w[0], 0.2)
    offs = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1)]
    xs, ys = [], []
    for k in range(inpn):
        dx, dy = offs[k % len(offs)]
        x, y = cx + dx, cy + dy
        w[k] = np.where((x >= 1) & (x <= nxin) & (y >= 1) & (y <= nyin), w[k], 0.0)
        xs.append(x)
        ys.append(y)
    w = w / w.sum(axis=0, keepdims=True)
    for k in range(inpn):
        x, y = xs[k], ys[k]
        ok = w[k] > 0
        inpx[k] = np.where(ok, x, 0)
        inpy[k] = np.where(ok, y, 0)
        inpa[k] = np.where(ok, (w[k] * grarea).astype(np.float32), 0.0)
    return nxin, nyin, inpx, inpy, inpa


def write_inpmat(path: str, nx: int, ny: int, i1seqx: np.ndarray, i1seqy: np.ndarray, inpx, inpy, inpa) -> None:
    """The input-matrix binary read by CMF_INPMAT_INIT_BIN (src/cmf_ctrl_forcing_mod.F90:418-458):
    3*INPN direct-access records of NX x NY 4-byte values (INPX int32, INPY int32, INPA float32),
    zero outside the sequence."""
    inpn = inpx.shape[0]
    with open(path, "wb") as f:
        for arr, dt in ((inpx, np.int32), (inpy, np.int32), (inpa, np.float32)):
            for k in range(inpn):
                g = np.zeros((ny, nx), dtype=dt)
                g[i1seqy - 1, i1seqx - 1] = arr[k]
                f.write(g.tobytes())


class DailyGammaRunoff:
    """i.i.d. Gamma(k=0.8, mean 2 mm/day) runoff per land cell per day (float32 mm/day)."""

    def __init__(self, ncell: int, seed: int, shape: float = 0.8, mean: float = 2.0, scale_mult: float = 1.0):
        self.rng = np.random.default_rng(seed + 1000003)
        self.ncell = ncell
        self.shape = shape
        self.theta = mean / shape * scale_mult

    def next(self) -> np.ndarray:
        return self.rng.gamma(self.shape, self.theta, size=self.ncell).astype(np.float32)


class AR1GammaRunoff:
    """Hourly runoff from a seeded AR(1) (phi=0.9) Gaussian process through a Gaussian copula
    with Gamma(k=0.8, theta=2.5 mm/day) marginals (float32 mm/day).  The Gamma quantile of the
    standard-normal value is read from a table built once (400,001 points on z in [-9, 9])."""

    _tables: dict = {}

    def __init__(self, ncell: int, seed: int, phi: float = 0.9, shape: float = 0.8, theta: float = 2.5):
        key = (shape, theta)
        if key not in AR1GammaRunoff._tables:
            from scipy.special import gammaincinv, ndtr

            z = np.linspace(-9.0, 9.0, 400001)
            u = np.clip(ndtr(z), 1e-300, 1.0 - 1e-16)
            AR1GammaRunoff._tables[key] = (z, gammaincinv(shape, u) * theta)
        self._z, self._q = AR1GammaRunoff._tables[key]
        self.rng = np.random.default_rng(seed + 2000003)
        self.phi = phi
        self.z = self.rng.standard_normal(ncell)

    def next(self) -> np.ndarray:
        eps = self.rng.standard_normal(self.z.shape[0])
        self.z = self.phi * self.z + np.sqrt(1.0 - self.phi * self.phi) * eps
        return np.interp(self.z, self._z, self._q).astype(np.float32)


# ----------------------------------------------------------------------------------------
# the configurations
# ----------------------------------------------------------------------------------------
def spec_config0(seed: int = 0) -> CaseSpec:
    """100x100 grid, 10,000 cells, 20 edge outlets; no bifurcation, levee or dam; daily forcing."""
    return CaseSpec(name="cfg0", nx=100, ny=100, land_frac=1.0, n_mouths=20, seed=seed,
                    dt=3600.0, ifrq_inp=24)


def spec_config1(seed: int = 1, scale: float = 1.0) -> CaseSpec:
    """1440x720 grid, ~300k land cells, 12k bifurcation channels x 5 levels, levees on 10% of
    cells, 2000 dams, hourly forcing.  ``scale`` shrinks the grid for parity-size runs."""
    nx = max(16, int(round(1440 * scale)))
    ny = max(8, int(round(720 * scale)))
    frac = 300000.0 / (1440 * 720)
    return CaseSpec(name="cfg1" if scale == 1.0 else f"cfg1s{scale:g}", nx=nx, ny=ny, land_frac=frac,
                    mouth_prob=0.1, seed=seed, lpthout=True,
                    npthout=max(4, int(round(12000 * scale * scale))), npthlev=5,
                    llevee=True, levee_frac=0.10, ldamout=True,
                    ndam=max(2, int(round(2000 * scale * scale))), dt=3600.0, ifrq_inp=1)


def spec_config2(n_domains: int = 8, n_min: int = 50_000, n_max: int = 2_000_000, seed: int = 11) -> list:
    """Regional domains of uneven size for the batched ensemble: `n_domains` networks with cell
    counts log-spaced from n_min to n_max, each generated with the config-1 laws (bifurcation
    channels, levees and dams in proportion to the cell count)."""
    sizes = np.geomspace(n_min, n_max, n_domains)
    specs = []
    for d, n in enumerate(sizes):
        sp = spec_config1(seed=seed + d, scale=float(np.sqrt(n / 300000.0)))
        sp.name = f"cfg2_d{d}"
        specs.append(sp)
    return specs



def spec_config4(seed: int = 4, scale: float = 1.0) -> CaseSpec:
    """7200x3600 grid, ~6M land cells (config-1 laws), 100k bifurcation channels x 5 levels, levees
    on 10% of cells, 10k dams, hourly forcing.  ``scale`` shrinks the grid (and the channel and dam
    counts with its area) for parity-size runs."""
    nx = max(16, int(round(7200 * scale)))
    ny = max(8, int(round(3600 * scale)))
    frac = 6_000_000.0 / (7200 * 3600)
    return CaseSpec(name="cfg4" if scale == 1.0 else f"cfg4s{scale:g}", nx=nx, ny=ny, land_frac=frac,
                    mouth_prob=0.1, seed=seed, lpthout=True,
                    npthout=max(4, int(round(100_000 * scale * scale))), npthlev=5,
                    llevee=True, levee_frac=0.10, ldamout=True,
                    ndam=max(2, int(round(10_000 * scale * scale))), dt=3600.0, ifrq_inp=1)
