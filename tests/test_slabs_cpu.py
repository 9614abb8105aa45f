"""The slab decomposition's host logic on the CPU (sc_lbm_b200/slabs.py).

Each slab is stepped by a stand-in domain that runs the CPU oracle on the
slab's own periodic lattice (its owned rows plus H ghost rows per side, as the
device domain does) and packs / unpacks halo rows in the library's buffer
layout.  After n steps with halos exchanged every k steps, the owned rows of
every slab must equal, bit for bit, the oracle run on the whole lattice:
* three slabs of uneven heights in one process (LocalRing over host buffers);
* ranks over gloo (DistRing): world size 2 (the two transfers to the same
  peer are told apart by their tags), 3 (distinct neighbours), and one rank
  exchanging with itself.
Porous lattice with walls, both solid interactions and a volume force.
"""
import ctypes
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

NX, NY = 24, 30
CASE = dict(fluid1=(0.8, 0.9, -0.15), fluid2=(1.2, 0.9, 0.15))


def _lattice():
    sys.path.insert(0, ROOT)
    from oracle import pyoracle
    from sc_lbm_b200 import workloads as W
    geom = [("walls", 1, "x"), ("circle", 7, 8, 10), ("circle", 5, 17, 21), ("square", 3, 5, 24)]
    mask, err = pyoracle.build_mask(NX, NY, geom)
    assert err == 0
    m = mask.astype(np.int32)
    N = NX * NY
    r1 = 1.0 + 0.05 * (2 * W.uniform(5, N) - 1)
    r2 = 0.7 + 0.05 * (2 * W.uniform(6, N) - 1)
    f = np.concatenate([W.populations(r1, m), W.populations(r2, m)])
    return m, f, list(W.force_vec(2e-4, "x"))


def _oracle_run(mask, nx, ny, f, steps, force):
    from oracle import pyoracle
    solids = [("solid_node", int(i % nx), int(i // nx)) for i in np.flatnonzero(mask == 0)]
    case = dict(nx=nx, ny=ny, geom=solids, mode="two", fluid1=CASE["fluid1"],
                fluid2=CASE["fluid2"], init=("file", f), force=(1, force), steps=steps)
    r = pyoracle.run_case(case)
    return np.concatenate([r["c1_f"], r["c2_f"]])


class OracleDomain:
    """Stand-in for a device Domain: the oracle steps the slab's lattice."""

    def __init__(self, nx, ny, mask, force):
        self.nx, self.ny, self.N = nx, ny, nx * ny
        self.mask, self.force = np.asarray(mask), force
        self.f = np.zeros(2 * 9 * self.N)

    def upload_f(self, comp, f):
        self.f[comp * 9 * self.N:(comp + 1) * 9 * self.N] = f

    def download_f(self, comp):
        return self.f[comp * 9 * self.N:(comp + 1) * 9 * self.N].copy()

    def step(self, n):
        self.f = _oracle_run(self.mask, self.nx, self.ny, self.f, n, self.force)

    def halo_bytes(self, H):
        return 2 * 9 * H * self.nx * 8

    def _rows(self, H, side, unpack):
        y = (self.ny - H if side else 0) if unpack else (self.ny - 2 * H if side else H)
        return slice(y, y + H)

    def halo_pack(self, H, side, ptr):
        f = self.f.reshape(2, 9, self.ny, self.nx)[:, :, self._rows(H, side, False), :]
        b = np.ascontiguousarray(f)
        ctypes.memmove(int(ptr), b.ctypes.data, b.nbytes)

    def halo_unpack(self, H, side, ptr):
        n = 2 * 9 * H * self.nx
        b = np.frombuffer((ctypes.c_double * n).from_address(int(ptr)), dtype=np.float64).copy()
        f = self.f.reshape(2, 9, self.ny, self.nx)
        f[:, :, self._rows(H, side, True), :] = b.reshape(2, 9, H, self.nx)

    # per-step exchange (sclbm_domain_halo_min_*): [component][9 slots][nx];
    # slots 0-5 whole-row values, 6-8 one value of each (crossing, bounce-back)
    # pair chosen by the mask of the receiving slab's first row across the cut
    ROW_UP, ROW_DOWN = [0, 1, 3, 2, 5, 6], [0, 1, 3, 4, 7, 8]
    LOW = [(2, 4, 0), (5, 7, -1), (6, 8, 1)]   # crossing into row 1, bounce-back in row 0
    UP = [(4, 2, 0), (7, 5, 1), (8, 6, -1)]    # crossing into row n, bounce-back in row n + 1
    CX = [0, 1, 0, -1, 0, 1, -1, -1, 1]

    def halo_min_bytes(self):
        return 2 * 9 * self.nx * 8

    def halo_min_pack(self, side, ptr):
        f = self.f.reshape(2, 9, self.ny, self.nx)
        m = np.asarray(self.mask).reshape(self.ny, self.nx) != 0
        n = self.ny - 2
        rows, pairs, rx, rb = (self.ROW_DOWN, self.UP, 0, 1) if side == 0 else \
            (self.ROW_UP, self.LOW, n + 1, n)
        b = np.zeros((2, 9, self.nx))
        b[:, :6] = f[:, rows, 1 if side == 0 else n, :]
        x = np.arange(self.nx)
        for p, (cross, bounce, shift) in enumerate(pairs):
            b[:, 6 + p] = np.where(m[rx], f[:, cross, rx, :], f[:, bounce, rb, (x + shift) % self.nx])
        ctypes.memmove(int(ptr), b.ctypes.data, b.nbytes)

    def halo_min_unpack(self, side, ptr):
        n = 2 * 9 * self.nx
        b = np.frombuffer((ctypes.c_double * n).from_address(int(ptr)), dtype=np.float64)
        b = b.reshape(2, 9, self.nx)
        f = self.f.reshape(2, 9, self.ny, self.nx)
        m = np.asarray(self.mask).reshape(self.ny, self.nx) != 0
        nn = self.ny - 2
        rows, pairs, ro, rg = (self.ROW_UP, self.LOW, 1, 0) if side == 0 else \
            (self.ROW_DOWN, self.UP, nn, nn + 1)
        f[:, rows, rg, :] = b[:, :6, :]
        x = np.arange(self.nx)
        for p, (cross, bounce, shift) in enumerate(pairs):
            v = b[:, 6 + p]
            take_cross = m[ro] & m[rg][(x - self.CX[cross]) % self.nx]
            f[:, cross, ro, :] = np.where(take_cross, v, f[:, cross, ro, :])
            solid = ~m[ro]
            tgt = (x + shift) % self.nx
            f[:, bounce, rg, tgt[solid]] = v[:, solid]

    def step_rows(self, row0, nrows, finish=False):
        """The step of rows [row0, row0 + nrows) only: each output slot (j, y)
        is taken from the full step when the row that writes it -- y - c_j
        for a fluid upstream node, else y (bounce-back) -- is in the range."""
        if not hasattr(self, "f_out"):
            self.f_out = np.zeros_like(self.f)
        full = _oracle_run(self.mask, self.nx, self.ny, self.f, 1, self.force).reshape(2, 9, self.ny,
                                                                                       self.nx)
        out = self.f_out.reshape(2, 9, self.ny, self.nx)
        m = np.asarray(self.mask).reshape(self.ny, self.nx) != 0
        CX = [0, 1, 0, -1, 0, 1, -1, -1, 1]
        CY = [0, 0, 1, 0, -1, 1, 1, -1, -1]
        y = np.arange(self.ny)[:, None] * np.ones((1, self.nx), int)
        inr = lambda r: (r >= row0) & (r < row0 + nrows)
        for j in range(9):
            up_fluid = np.roll(np.roll(m, CY[j], 0), CX[j], 1)
            src = np.where(up_fluid, (y - CY[j]) % self.ny, y)
            take = inr(src) & m
            out[:, j][:, take] = full[:, j][:, take]
            out[:, j][:, ~m] = 0.0
        if finish:
            self.f, self.f_out = self.f_out, self.f


def _slab(mask, f, force, y0, y1, k, per_step=False):
    from sc_lbm_b200 import slabs
    s = slabs.Slab(NX, NY, mask, y0, y1, k, per_step=per_step,
                   make_domain=lambda nx, ny, m: OracleDomain(nx, ny, m, force))
    s.upload_f(0, f[:9 * NX * NY])
    s.upload_f(1, f[9 * NX * NY:])
    return s


def _owned_want(want, y0, y1):
    w = want.reshape(2, 9, NY, NX)
    return [w[c][:, y0:y1, :] for c in range(2)]


def test_partition():
    from sc_lbm_b200.slabs import partition
    assert partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert partition(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        partition(2, 3)


@pytest.mark.parametrize("k,steps", [(1, 5), (2, 5), (3, 6)])
def test_local_ring_matches_whole_lattice(k, steps):
    from sc_lbm_b200 import slabs
    mask, f, force = _lattice()
    want = _oracle_run(mask, NX, NY, f, steps, force)
    cuts = [(0, 7), (7, 19), (19, 30)]
    ss = [_slab(mask, f, force, y0, y1, k) for y0, y1 in cuts]
    slabs.run(ss, slabs.LocalRing(ss, device="cpu"), steps)
    for s, (y0, y1) in zip(ss, cuts):
        for c, w in enumerate(_owned_want(want, y0, y1)):
            assert np.array_equal(s.owned_f(c), w), (y0, c)


@pytest.mark.parametrize("overlap", [False, True])
def test_per_step_exchange_matches_whole_lattice(overlap):
    """One ghost row per side and nine values per component and column per
    side each step (the six the neighbour cannot compute, the three that
    crossed the cut): owned rows equal the whole-lattice run bit for bit,
    also when the rows away from the cuts are stepped before the exchange."""
    from sc_lbm_b200 import slabs
    mask, f, force = _lattice()
    steps = 5
    want = _oracle_run(mask, NX, NY, f, steps, force)
    cuts = [(0, 7), (7, 19), (19, 30)]
    ss = [_slab(mask, f, force, y0, y1, 1, per_step=True) for y0, y1 in cuts]
    assert ss[0].H == 1 and ss[0].halo_bytes() == 2 * 9 * NX * 8
    slabs.run(ss, slabs.LocalRing(ss, device="cpu"), steps, overlap=overlap)
    for s, (y0, y1) in zip(ss, cuts):
        for c, w in enumerate(_owned_want(want, y0, y1)):
            assert np.array_equal(s.owned_f(c), w), (overlap, y0, c)


def test_per_step_exchange_is_sharp():
    """Without the three crossing / bounce-back values the rows at the cuts go
    wrong: the exchange carries nothing superfluous."""
    from sc_lbm_b200 import slabs
    mask, f, force = _lattice()
    want = _oracle_run(mask, NX, NY, f, 3, force)
    cuts = [(0, 15), (15, 30)]
    ss = [_slab(mask, f, force, y0, y1, 1, per_step=True) for y0, y1 in cuts]
    for s in ss:
        s.domain.LOW = s.domain.UP = []
    slabs.run(ss, slabs.LocalRing(ss, device="cpu"), 3)
    assert not all(np.array_equal(s.owned_f(c), w) for s, (y0, y1) in zip(ss, cuts)
                   for c, w in enumerate(_owned_want(want, y0, y1)))


def test_slab_too_thin_is_refused():
    mask, f, force = _lattice()
    with pytest.raises(ValueError):
        _slab(mask, f, force, 0, 3, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, steps, k, q, per_step=False, overlap=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from sc_lbm_b200 import slabs
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mask, f, force = _lattice()
        want = _oracle_run(mask, NX, NY, f, steps, force)
        y0, y1 = slabs.partition(NY, world)[rank]
        s = _slab(mask, f, force, y0, y1, k, per_step=per_step)
        slabs.run([s], slabs.DistRing(s, device="cpu"), steps, overlap=overlap)
        ok = all(np.array_equal(s.owned_f(c), w) for c, w in enumerate(_owned_want(want, y0, y1)))
        dist.barrier()
    finally:
        dist.destroy_process_group()
    q.put((rank, ok))


@pytest.mark.parametrize("world,per_step", [(1, False), (2, False), (3, False), (2, True), (3, True)])
def test_dist_ring_gloo(world, per_step):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 4, 2, q, per_step, per_step))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(world))
    assert got == [(r, True) for r in range(world)]


def test_too_few_ghost_rows_break_parity():
    """The check is sharp: two steps between exchanges with the ghost rows of
    one step (H = 2) corrupt the owned rows next to every cut."""
    from sc_lbm_b200 import slabs
    mask, f, force = _lattice()
    want = _oracle_run(mask, NX, NY, f, 4, force)
    cuts = [(0, 15), (15, 30)]
    ss = [_slab(mask, f, force, y0, y1, 1) for y0, y1 in cuts]
    for s in ss:
        s.k = 2
    slabs.run(ss, slabs.LocalRing(ss, device="cpu"), 4)
    assert not all(np.array_equal(s.owned_f(c), w) for s, (y0, y1) in zip(ss, cuts)
                   for c, w in enumerate(_owned_want(want, y0, y1)))
