"""GPU checks of the slab decomposition (sc_lbm_b200/slabs.py, slab.cu).

* Three slabs of uneven heights on one GPU, halos exchanged through device
  buffers (LocalRing) every k steps: the owned rows equal the same rows of one
  domain holding the whole lattice, byte for byte, in every storage precision
  (FP64 therefore bit-identical to the reference), on a porous lattice with
  walls, solid interactions and a volume force;
* the halo entry points refuse bad arguments;
* a one-rank NCCL ring on the library's own stream equals the whole lattice;
* the torchrun driver (one rank, NCCL process group, the exchange with
  itself) runs and reports its line.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lattice(sclbm):
    from sc_lbm_b200 import workloads as W
    nx, ny = 200, 90
    m, _, _ = W.disk_mask(nx, ny, 0.75, 3, 7, seed=17, walls="x")
    N = nx * ny
    r1 = 1.0 + 0.02 * (2 * W.uniform(41, N) - 1)
    r2 = 0.6 + 0.02 * (2 * W.uniform(42, N) - 1)
    p = sclbm.make_params(ncomp=2, tau=(0.8, 1.1), g_fluid=(0.9, 0.9), g_solid=(-0.2, 0.2),
                          rho_ref=(1.0, 0.6), force=(W.force_vec(1e-5, "x"), None))
    return nx, ny, m, p, W.populations(r1, m), W.populations(r2, m)


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"])
@pytest.mark.parametrize("k", [1, 3])
def test_slabs_on_one_gpu_match_whole_lattice(sclbm, prec_name, k):
    from sc_lbm_b200 import slabs
    prec = getattr(sclbm, prec_name)
    nx, ny, m, p, f1, f2 = _lattice(sclbm)
    whole = sclbm.Domain(nx, ny, m, p, prec)
    whole.upload_f(0, f1)
    whole.upload_f(1, f2)
    steps = 25
    whole.step(steps)
    cuts = [(0, 17), (17, 60), (60, 90)]
    ss = [slabs.Slab(nx, ny, m, y0, y1, k, params=p, precision=prec) for y0, y1 in cuts]
    for s in ss:
        s.upload_f(0, f1)
        s.upload_f(1, f2)
    slabs.run(ss, slabs.LocalRing(ss), steps)
    for c in range(2):
        w = whole.download_f(c).reshape(9, ny, nx)
        for s, (y0, y1) in zip(ss, cuts):
            assert s.owned_f(c).tobytes() == np.ascontiguousarray(w[:, y0:y1, :]).tobytes(), (y0, c)


@pytest.mark.parametrize("prec_name", ["FP64", "FP32_SHIFTED", "FP16_SHIFTED"])
@pytest.mark.parametrize("overlap", [False, True])
def test_per_step_slabs_match_whole_lattice(sclbm, prec_name, overlap):
    """One ghost row per side, nine values per component and column per side
    each step (sclbm_domain_halo_min_*), with the rows away from the cuts
    stepped before the exchange when `overlap` (sclbm_domain_step_rows): the
    owned rows equal one domain holding the lattice, byte for byte."""
    from sc_lbm_b200 import slabs
    prec = getattr(sclbm, prec_name)
    nx, ny, m, p, f1, f2 = _lattice(sclbm)
    whole = sclbm.Domain(nx, ny, m, p, prec)
    whole.upload_f(0, f1)
    whole.upload_f(1, f2)
    steps = 25
    whole.step(steps)
    cuts = [(0, 17), (17, 60), (60, 90)]
    ss = [slabs.Slab(nx, ny, m, y0, y1, params=p, precision=prec, per_step=True) for y0, y1 in cuts]
    es = {sclbm.FP64: 8, sclbm.FP32_SHIFTED: 4, sclbm.FP16_SHIFTED: 2}[prec]
    assert ss[0].halo_bytes() == 2 * 9 * nx * es
    for s in ss:
        s.upload_f(0, f1)
        s.upload_f(1, f2)
    slabs.run(ss, slabs.LocalRing(ss), steps, overlap=overlap)
    for c in range(2):
        w = whole.download_f(c).reshape(9, ny, nx)
        for s, (y0, y1) in zip(ss, cuts):
            assert s.owned_f(c).tobytes() == np.ascontiguousarray(w[:, y0:y1, :]).tobytes(), \
                (overlap, y0, c)


def test_step_rows_in_pieces_equals_one_step(sclbm):
    """Stepping a domain's rows in three pieces and finishing equals one step."""
    nx, ny, m, p, f1, f2 = _lattice(sclbm)
    for prec in (sclbm.FP64, sclbm.FP32_SHIFTED):
        a = sclbm.Domain(nx, ny, m, p, prec)
        b = sclbm.Domain(nx, ny, m, p, prec)
        for d in (a, b):
            d.upload_f(0, f1)
            d.upload_f(1, f2)
        a.step(2)
        for _ in range(2):
            b.step_rows(0, 31)
            b.step_rows(60, 30)
            b.step_rows(31, 29, finish=True)
        for c in range(2):
            assert a.download_f(c).tobytes() == b.download_f(c).tobytes()
    with pytest.raises(IndexError):
        b.step_rows(80, 20)


def test_dist_ring_one_rank_nccl_on_the_library_stream(sclbm, tmp_path):
    """DistRing over an NCCL group of one rank while the library keeps its own
    stream (no set_stream): the exchange orders the library's copies and
    torch's stream, and the slab equals the whole lattice byte for byte."""
    import torch
    import torch.distributed as dist
    from sc_lbm_b200 import slabs
    nx, ny, m, p, f1, f2 = _lattice(sclbm)
    whole = sclbm.Domain(nx, ny, m, p, sclbm.FP32_SHIFTED)
    whole.upload_f(0, f1)
    whole.upload_f(1, f2)
    whole.step(9)
    store = dist.FileStore(str(tmp_path / "store"), 1)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        s = slabs.Slab(nx, ny, m, 0, ny, 2, params=p, precision=sclbm.FP32_SHIFTED)
        s.upload_f(0, f1)
        s.upload_f(1, f2)
        slabs.run([s], slabs.DistRing(s), 9)
        torch.cuda.synchronize()
        for c in range(2):
            assert s.owned_f(c).tobytes() == whole.download_f(c).tobytes()
    finally:
        dist.destroy_process_group()


def test_halo_arguments(sclbm):
    import torch
    nx, ny, m, p, f1, f2 = _lattice(sclbm)
    d = sclbm.Domain(nx, 12, m[:nx * 12], p, sclbm.FP32_SHIFTED)
    assert d.halo_bytes(2) == 2 * 9 * 2 * nx * 4
    buf = torch.empty(d.halo_bytes(4), dtype=torch.uint8, device="cuda")
    d.halo_pack(4, 0, buf.data_ptr())           # 3 * 4 rows fit in 12
    with pytest.raises(IndexError):
        d.halo_pack(5, 0, buf.data_ptr())       # 15 > 12
    with pytest.raises(ValueError):
        d.halo_unpack(2, 2, buf.data_ptr())
    with pytest.raises(ValueError):
        d.halo_pack(2, 0, 0)


def test_driver_under_torchrun_one_rank():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=1",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "-m", "sc_lbm_b200.slabs",
           "--nx", "1024", "--rows-per-rank", "512", "--steps", "20", "--warmup", "3"]
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("{")]
    d = json.loads(line[-1])
    assert d["slabs"] == 1 and d["halo_rows"] == 2 and d["mlups"] > 0
