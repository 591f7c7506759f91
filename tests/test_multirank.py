"""Multi-rank paths on CPU (gloo, world size 2) and the split stage/sub-step API on one GPU.

Basin regions (cmf_b200.regions) are closed under I1NEXT and bifurcation, so ranks exchange only
the 8-byte MIN of DT_MIN per outer step (CMF_MPI_ADPSTP, src/cmf_ctrl_mpi_mod.F90:261-281); the
regional run must equal the whole-domain run bit for bit."""
from __future__ import annotations

import datetime
import math
import os
import socket

import numpy as np
import pytest

NSTEPS = 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _grid_runoff(nx, ny, k):
    rng = np.random.default_rng(1000 + k)
    g = rng.gamma(0.8, 2.5, size=nx * ny).astype(np.float32).astype(np.float64)
    return g * 6.0


def _region_worker(rank, world, port, region_dirs, out_dir):
    import torch
    import torch.distributed as dist
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "cama-flood_v4_b200"), os.path.join(root, "oracle")]
    from oracle import Oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    o = Oracle(region_dirs[rank])
    nts = []
    for k in range(NSTEPS):
        o.put_runoff_map(_grid_runoff(o.nx, o.ny, k))
        local = o.stage()
        t = torch.tensor([local], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        nt, dt = o.substeps(float(t.item()))
        nts.append((nt, dt))
    gx, gy = o.i("i1seqx"), o.i("i1seqy")
    flat = (gy - 1) * o.nx + (gx - 1)
    grids = {}
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto"):
        g = np.full(o.nx * o.ny, np.nan)
        g[flat] = o.d(f)
        grids[f] = g
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), nts=np.array(nts), **grids)
    dist.barrier()
    dist.destroy_process_group()


def test_regions_partition_and_balance(case_dirs, tmp_path):
    from cmf_b200 import regions

    dirs = regions.split_case(case_dirs["cfg1s"], 2, str(tmp_path))
    reg = np.fromfile(os.path.join(dirs[0], "mpireg.bin"), dtype="<i4")
    land = reg != regions.IMIS
    counts = [int(np.sum(reg == r)) for r in (1, 2)]
    assert sum(counts) == int(land.sum()) and min(counts) > 0.3 * max(counts)
    # every bifurcation channel stays inside one region
    with open(os.path.join(dirs[0], "diminfo.txt")) as f:
        nx = int(f.readline().split()[0])
    for ix, iy, jx, jy in regions.read_bif_pairs(case_dirs["cfg1s"]):
        assert reg[(iy - 1) * nx + ix - 1] == reg[(jy - 1) * nx + jx - 1]


def test_gloo_regions_equal_whole_domain(case_dirs, tmp_path):
    import torch.multiprocessing as mp

    from cmf_b200 import regions
    from oracle import Oracle

    dirs = regions.split_case(case_dirs["cfg1s"], 2, str(tmp_path))
    mp.start_processes(_region_worker, args=(2, _free_port(), dirs, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    whole = Oracle(case_dirs["cfg1s"])
    ref_nt = []
    for k in range(NSTEPS):
        whole.put_runoff_map(_grid_runoff(whole.nx, whole.ny, k))
        ref_nt.append(whole.advance())
    gx, gy = whole.i("i1seqx"), whole.i("i1seqy")
    flat = (gy - 1) * whole.nx + (gx - 1)
    parts = [dict(np.load(os.path.join(str(tmp_path), f"rank{r}.npz"))) for r in (0, 1)]
    for p in parts:
        assert [tuple(x) for x in p["nts"]] == [(int(a), float(b)) for a, b in ref_nt]
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto"):
        merged = np.where(np.isnan(parts[0][f]), parts[1][f], parts[0][f])[flat]
        assert np.array_equal(merged.view(np.int64), whole.d(f).view(np.int64)), f


def _member_worker(rank, world, port, nmembers, out_dir):
    import torch
    import torch.distributed as dist
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "cama-flood_v4_b200")]
    from cmf_b200.regions import members_for_rank

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = torch.zeros(nmembers, dtype=torch.int64)
    for m in members_for_rank(nmembers, world, rank):
        mine[m] += 1
    dist.all_reduce(mine)
    np.save(os.path.join(out_dir, f"members{rank}.npy"), mine.numpy())
    dist.destroy_process_group()


@pytest.mark.parametrize("nmembers", [7, 64])
def test_gloo_member_sharding_covers_every_member_once(tmp_path, nmembers):
    import torch.multiprocessing as mp

    mp.start_processes(_member_worker, args=(2, _free_port(), nmembers, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in (0, 1):
        assert np.all(np.load(os.path.join(str(tmp_path), f"members{r}.npy")) == 1)


def _units_worker(rank, world, port, loads, nmembers, out_dir):
    import torch
    import torch.distributed as dist
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "cama-flood_v4_b200")]
    from cmf_b200.regions import pack_units

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = torch.zeros(len(loads), nmembers, dtype=torch.int64)
    load = torch.zeros(world, dtype=torch.float64)
    for d, ms in enumerate(pack_units(loads, nmembers, world)[rank]):     # each rank packs on its own
        for m in ms:
            mine[d, m] += 1
            load[rank] += loads[d]
    dist.all_reduce(mine)
    dist.all_reduce(load)
    np.save(os.path.join(out_dir, f"units{rank}.npy"), mine.numpy())
    np.save(os.path.join(out_dir, f"loads{rank}.npy"), load.numpy())
    dist.destroy_process_group()


def test_gloo_domain_member_packing_covers_every_unit_once(tmp_path):
    """Members x domains of uneven size over two gloo ranks (the config-2 partition): each rank
    packs independently, every (domain, member) unit is owned exactly once, and the ranks' loads
    (cells x expected NT) differ by at most the largest unit."""
    import torch.multiprocessing as mp

    loads = [49424 * 24, 84124 * 25, 142834 * 25, 241678 * 26, 410196 * 30, 695486 * 30, 1177949 * 33, 1997245 * 45]
    mp.start_processes(_units_worker, args=(2, _free_port(), loads, 7, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in (0, 1):
        assert np.all(np.load(os.path.join(str(tmp_path), f"units{r}.npy")) == 1)
        ld = np.load(os.path.join(str(tmp_path), f"loads{r}.npy"))
        assert ld.sum() == 7 * sum(loads) and ld.max() - ld.min() <= max(loads)


def test_pack_units_and_expected_nt():
    from cmf_b200.regions import expected_nt, pack_units

    loads = [5.0, 3.0, 3.0, 1.0]
    for world in (1, 2, 3, 5, 40):
        owned = pack_units(loads, 6, world)
        seen = sorted((d, m) for per in owned for d, ms in enumerate(per) for m in ms)
        assert seen == [(d, m) for d in range(4) for m in range(6)]
        acc = [sum(len(ms) * loads[d] for d, ms in enumerate(per)) for per in owned]
        assert max(acc) <= sum(loads) * 6 / world + max(loads)
        assert all(ms == sorted(ms) for per in owned for ms in per)
    assert pack_units(loads, 6, 2) == pack_units(list(loads), 6, 2)            # deterministic
    # CALC_ADPSTP on a half-full channel: the key of the shortest, deepest reach decides NT
    dst = np.array([12000.0, 3000.0, 8000.0, 50000.0])
    hgt = np.array([4.0, 9.0, 2.0, 6.0])
    keys = [(0.7 * d) * math.pow(9.8 * max(h * 0.5, 0.01), -0.5) for d, h in zip(dst[:3], hgt[:3])]
    keys.append((0.7 * 10000.0) * math.pow(9.8 * 3.0, -0.5))                 # the mouth: PDSTMTH
    dt_min = min([3600.0] + keys)
    assert expected_nt(dst, hgt, 3) == int(3600.0 * (1.0 / dt_min) - float(np.float32(0.01))) + 1 == 12


@pytest.mark.gpu
def test_gpu_regions_with_host_min_equal_whole_domain(case_dirs, tmp_path):
    """Two regional GPU contexts, DT_MIN reduced on the host between cmf_gpu_ctx_stage and
    cmf_gpu_ctx_substeps, reproduce the whole-domain GPU context bit for bit."""
    from cmf_b200 import HostModel, PhysicsGPU, regions

    dirs = regions.split_case(case_dirs["cfg1s"], 2, str(tmp_path))
    hw = HostModel(case_dirs["cfg1s"])
    gw = PhysicsGPU(hw)
    hs = [HostModel(d) for d in dirs]
    gs = [PhysicsGPU(h) for h in hs]
    for k in range(NSTEPS):
        grid = _grid_runoff(hw.nx, hw.ny, k)
        gw.put_runoff(hw.conv_resol(grid))
        ntw, dtw, _ = gw.advance()
        local = []
        for h, g in zip(hs, gs):
            g.put_runoff(h.conv_resol(grid))
            local.append(g.stage()[0])
        dtmin = min(local)
        for g in gs:
            nt, dt, _ = g.substeps(dtmin)
            assert nt[0] == ntw[0] and dt[0] == dtw[0]
    flat_w = (hw.i1seqy - 1) * hw.nx + (hw.i1seqx - 1)
    sw = gw.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto"):
        g = np.full(hw.nx * hw.ny, np.nan)
        for h, p in zip(hs, gs):
            g[(h.i1seqy - 1) * h.nx + (h.i1seqx - 1)] = p.get_state()[f][0]
        assert np.array_equal(g[flat_w].view(np.int64), sw[f][0].view(np.int64)), f


def _gpu_region_worker(rank, world, port, region_dirs, out_dir):
    """One rank of the product's split outer step: cmf_gpu_ctx_stage -> 8-byte MIN all-reduce over
    gloo (CMF_MPI_ADPSTP, src/cmf_ctrl_mpi_mod.F90:261-281) -> cmf_gpu_ctx_substeps."""
    import torch
    import torch.distributed as dist
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [os.path.join(root, "cama-flood_v4_b200")]
    from cmf_b200 import HostModel, PhysicsGPU

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    h = HostModel(region_dirs[rank])
    g = PhysicsGPU(h, device=0)
    nts = []
    for k in range(NSTEPS):
        g.put_runoff(h.conv_resol(_grid_runoff(h.nx, h.ny, k)))
        local = float(g.stage()[0])
        t = torch.tensor([local], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        nt, dt, _ = g.substeps(float(t.item()))
        nts.append((int(nt[0]), float(dt[0])))
    flat = (h.i1seqy - 1) * h.nx + (h.i1seqx - 1)
    st = g.get_state()
    grids = {}
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto"):
        a = np.full(h.nx * h.ny, np.nan)
        a[flat] = st[f][0]
        grids[f] = a
    np.savez(os.path.join(out_dir, f"gpu_rank{rank}.npz"), nts=np.array(nts), **grids)
    g.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_gloo_two_ranks_product_split_equal_whole_domain(case_dirs, tmp_path):
    """World size 2 over gloo, both ranks on the one GPU (their kernels never wait on each other;
    the only exchange is the host-side MIN of DT_MIN): the product's split API per rank reproduces
    the whole-domain GPU run bit for bit, NT and DT included."""
    import torch.multiprocessing as mp

    from cmf_b200 import HostModel, PhysicsGPU, regions

    dirs = regions.split_case(case_dirs["cfg1s"], 2, str(tmp_path))
    mp.start_processes(_gpu_region_worker, args=(2, _free_port(), dirs, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    hw = HostModel(case_dirs["cfg1s"])
    gw = PhysicsGPU(hw)
    ref = []
    for k in range(NSTEPS):
        gw.put_runoff(hw.conv_resol(_grid_runoff(hw.nx, hw.ny, k)))
        nt, dt, _ = gw.advance()
        ref.append((int(nt[0]), float(dt[0])))
    parts = [dict(np.load(os.path.join(str(tmp_path), f"gpu_rank{r}.npz"))) for r in (0, 1)]
    for p in parts:
        assert [(int(a), float(b)) for a, b in p["nts"]] == ref
    flat = (hw.i1seqy - 1) * hw.nx + (hw.i1seqx - 1)
    sw = gw.get_state()
    for f in ("rivsto", "fldsto", "rivout", "fldout", "levsto", "damsto"):
        merged = np.where(np.isnan(parts[0][f]), parts[1][f], parts[0][f])[flat]
        assert np.array_equal(merged.view(np.int64), sw[f][0].view(np.int64)), f
