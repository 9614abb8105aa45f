"""Slab decomposition: one lattice cut into row slabs, one slab per GPU (or
several slabs on one GPU), with halo rows exchanged between steps.

    torchrun --nproc-per-node N -m sc_lbm_b200.slabs [--nx 4096] [--rows-per-rank 4096]
             [--steps 200] [--halo-steps 1] [--precision fp32]

A slab owning global rows [y0, y1) is a device ``Domain`` of
y1 - y0 + 2H rows: H ghost rows copied from the slab below and H from the
slab above (periodic across the lattice).  With H = 2k the owned rows stay
exact for k fused steps; then every slab sends its first H owned rows down
and its last H owned rows up, and receives its ghost rows (the halo
entry points of include/sclbm.h, slab.cu).  Owned rows are bit-identical to
stepping the whole lattice in one domain.  This is the slab scheme of the
reference's MATLAB generator (tests/lbm/lbm_matlab/two_phase_flow/
main_droplet.m:162-465), which exchanges the three crossing populations and a
density row per step; whole population rows keep the exchange a plain copy
of contiguous rows and let k steps run between exchanges.

Per-step mode (``per_step=True``): one ghost row per side, exchanged after
every step, nine values per component and column per side -- the six
populations of the row next to the cut that the neighbour cannot compute and
the three that crossed the cut -- half of what the whole-row halo moves per
step (18), still bit-identical.  Rows two or more away from a cut need nothing
from the exchange, so ``run(..., overlap=True)`` steps them while the halo is
in flight and the three rows at each cut afterwards (sclbm_domain_step_rows).
A 4096-wide FP32 slab then exchanges 2 x 295 KB per step.

Transports: ``LocalRing`` for slabs held by one process (device copies in
stream order) and ``DistRing`` for one slab per rank (torch.distributed
point-to-point: NCCL over NVLink between GPUs, gloo for host tensors; NCCL
runs on torch's stream, so the interior rows stepped on the library stream
before it overlap with the transfer).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def partition(ny: int, parts: int) -> list[tuple[int, int]]:
    """Rows [y0, y1) of each slab: as even as possible, the first ny % parts
    slabs one row taller."""
    if parts < 1 or ny < parts:
        raise ValueError("need 1 <= parts <= ny")
    base, extra = divmod(ny, parts)
    out, y = [], 0
    for r in range(parts):
        h = base + (1 if r < extra else 0)
        out.append((y, y + h))
        y += h
    return out


class Slab:
    """The domain of one slab: global rows [y0, y1) plus H = 2 * halo_steps
    ghost rows on each side, cut from the lattice's mask (periodic in y).

    ``domain`` is a ``Domain`` (or any object with its step / halo_* /
    upload_f / download_f methods, which the host-side tests use)."""

    def __init__(self, nx, ny, mask, y0, y1, halo_steps=1, make_domain=None, params=None,
                 precision=None, per_step=False):
        self.nx, self.ny, self.y0, self.y1 = int(nx), int(ny), int(y0), int(y1)
        self.per_step = bool(per_step)
        self.k = 1 if self.per_step else int(halo_steps)
        self.H = 1 if self.per_step else 2 * self.k
        if self.k < 1:
            raise ValueError("halo_steps >= 1")
        if self.y1 - self.y0 < max(self.H, 1):
            raise ValueError("a slab needs at least 2 * halo_steps rows of its own")
        self.rows = np.arange(self.y0 - self.H, self.y1 + self.H) % self.ny
        m = np.asarray(mask, dtype=np.int32).reshape(self.ny, self.nx)[self.rows].ravel()
        if make_domain is None:
            from .api import Domain
            self.domain = Domain(self.nx, len(self.rows), m, params, precision)
        else:
            self.domain = make_domain(self.nx, len(self.rows), m)

    @property
    def owned(self) -> int:
        return self.y1 - self.y0

    def upload_f(self, comp: int, f_global: np.ndarray) -> None:
        """Populations of the whole lattice ([9 N] reference layout) -> this
        slab's rows, ghosts included."""
        f = np.asarray(f_global, dtype=np.float64).reshape(9, self.ny, self.nx)[:, self.rows, :]
        self.domain.upload_f(comp, np.ascontiguousarray(f).ravel())

    def owned_f(self, comp: int) -> np.ndarray:
        """[9, y1 - y0, nx] populations of the owned rows."""
        f = self.domain.download_f(comp).reshape(9, len(self.rows), self.nx)
        return f[:, self.H:self.H + self.owned, :]

    def halo_bytes(self) -> int:
        return self.domain.halo_min_bytes() if self.per_step else self.domain.halo_bytes(self.H)

    def pack(self, side: int, ptr: int) -> None:
        if self.per_step:
            self.domain.halo_min_pack(side, ptr)
        else:
            self.domain.halo_pack(self.H, side, ptr)

    def unpack(self, side: int, ptr: int) -> None:
        if self.per_step:
            self.domain.halo_min_unpack(side, ptr)
        else:
            self.domain.halo_unpack(self.H, side, ptr)

    # per-step mode: domain rows 0 and n-1 are the ghost rows; the exchange
    # writes rows 0, 1, n-2 and n-1, and a row's step reads the densities of
    # its neighbours, so rows [3, n-3) need nothing from it
    def step_interior(self) -> None:
        n = len(self.rows)
        if n > 6:
            self.domain.step_rows(3, n - 6, finish=False)

    def step_boundary(self) -> None:
        n = len(self.rows)
        if n > 6:
            self.domain.step_rows(0, 3, finish=False)
            self.domain.step_rows(n - 3, 3, finish=True)
        else:
            self.domain.step_rows(0, n, finish=True)


class LocalRing:
    """Slabs of one lattice held by this process, in order from y = 0; halos
    go through device buffers in the library's stream order."""

    def __init__(self, slabs, device="cuda"):
        import torch
        self.slabs = list(slabs)
        nb = self.slabs[0].halo_bytes()
        self.low = [torch.empty(nb, dtype=torch.uint8, device=device) for _ in self.slabs]
        self.up = [torch.empty(nb, dtype=torch.uint8, device=device) for _ in self.slabs]

    def exchange(self) -> None:
        n = len(self.slabs)
        for s, lo, up in zip(self.slabs, self.low, self.up):
            s.pack(0, lo.data_ptr())
            s.pack(1, up.data_ptr())
        for r, s in enumerate(self.slabs):
            s.unpack(0, self.up[(r - 1) % n].data_ptr())   # rows below: the last rows of r-1
            s.unpack(1, self.low[(r + 1) % n].data_ptr())  # rows above: the first rows of r+1


class DistRing:
    """One slab per rank of a torch.distributed group, rank r owning the r-th
    slab from y = 0.  Each exchange sends the first H owned rows to rank r-1
    (tag 0) and the last H to rank r+1 (tag 1), all four transfers in one
    batch (NCCL groups them; gloo runs them asynchronously)."""

    def __init__(self, slab, group=None, device="cuda"):
        import torch
        import torch.distributed as dist
        self.dist, self.group = dist, group
        self.slab = slab
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        nb = slab.halo_bytes()
        self.bufs = {k: torch.empty(nb, dtype=torch.uint8, device=device)
                     for k in ("send_low", "send_up", "recv_low", "recv_up")}
        self.torch = torch
        self.cuda = torch.device(device).type == "cuda"

    def _library_stream(self):
        """The stream the library queues its copies on (torch's own streams
        order the transfers): each waits for the other around the exchange."""
        from .capi import lib
        ptr = lib().sclbm_get_stream()
        return self.torch.cuda.ExternalStream(ptr) if ptr else None

    def _peer(self, r):
        g = r % self.world
        return g if self.group is None else self.dist.get_global_rank(self.group, g)

    def exchange(self) -> None:
        b, s = self.bufs, self.slab
        s.pack(0, b["send_low"].data_ptr())
        s.pack(1, b["send_up"].data_ptr())
        lib_stream = self._library_stream() if self.cuda else None
        if lib_stream is not None:
            self.torch.cuda.current_stream().wait_stream(lib_stream)
        if self.world == 1:
            b["recv_low"].copy_(b["send_up"])
            b["recv_up"].copy_(b["send_low"])
        else:
            d = self.dist
            prev, nxt = self._peer(self.rank - 1), self._peer(self.rank + 1)
            ops = [d.P2POp(d.isend, b["send_low"], prev, self.group, 0),
                   d.P2POp(d.isend, b["send_up"], nxt, self.group, 1),
                   d.P2POp(d.irecv, b["recv_up"], nxt, self.group, 0),
                   d.P2POp(d.irecv, b["recv_low"], prev, self.group, 1)]
            for req in d.batch_isend_irecv(ops):
                req.wait()
        if lib_stream is not None:
            lib_stream.wait_stream(self.torch.cuda.current_stream())
        s.unpack(0, b["recv_low"].data_ptr())
        s.unpack(1, b["recv_up"].data_ptr())


def run(slabs, transport, steps: int, overlap: bool = False) -> None:
    """Advance every slab `steps` steps, exchanging halos every k steps.  In
    per-step mode with `overlap`, each step runs the rows that need no halo,
    then the exchange of the previous step's boundary values, then the rows
    at the cuts (the exchange of the first step finds the state already
    consistent and changes nothing); a last exchange completes the owned rows."""
    if slabs[0].per_step and overlap:
        for _ in range(int(steps)):
            for s in slabs:
                s.step_interior()
            transport.exchange()
            for s in slabs:
                s.step_boundary()
        if steps > 0:
            transport.exchange()
        return
    k = slabs[0].k
    left = int(steps)
    while left > 0:
        n = min(k, left)
        for s in slabs:
            s.domain.step(n)
        transport.exchange()
        left -= n


# ----------------------------------------------------------------------------- driver
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=4096)
    ap.add_argument("--rows-per-rank", type=int, default=4096)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--halo-steps", type=int, default=1)
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "fp16"])
    ap.add_argument("--per-step", action="store_true",
                    help="one ghost row, nine values per column and component per side every step, "
                         "the exchange overlapped with the rows away from the cuts")
    args = ap.parse_args()

    import torch
    import torch.distributed as dist
    import sc_lbm_b200 as sc
    from datetime import timedelta

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29531")
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=timedelta(seconds=120),
                            device_id=torch.device("cuda", local))
    sc.set_stream(torch.cuda.current_stream().cuda_stream)
    prec = {"fp64": sc.FP64, "fp32": sc.FP32_SHIFTED, "fp16": sc.FP16_SHIFTED}[args.precision]
    nx, ny = args.nx, args.rows_per_rank * world
    y0, y1 = partition(ny, world)[rank]
    params = sc.make_params(ncomp=2, g_fluid=(1.2, 1.2), rho_ref=(1.0, 1.0))
    slab = Slab(nx, ny, np.ones(nx * ny, np.int32), y0, y1, args.halo_steps, params=params,
                precision=prec, per_step=args.per_step)
    # spinodal-type state seeded on the device (per slab, not the global field)
    slab.domain.init_noise(0, 1.0, 0.01, 101 + 2 * rank)
    slab.domain.init_noise(1, 1.0, 0.01, 102 + 2 * rank)
    ring = DistRing(slab)
    run([slab], ring, args.warmup, overlap=args.per_step)
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run([slab], ring, args.steps, overlap=args.per_step)
    e1.record()
    torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_step = float(ms.item()) / args.steps
    if rank == 0:
        print(json.dumps({"slabs": world, "lattice": [nx, ny], "precision": args.precision,
                          "halo_rows": slab.H, "halo_bytes_per_side": slab.halo_bytes(),
                          "per_step": args.per_step,
                          "ms_per_step": round(ms_step, 5),
                          "mlups": round(nx * ny / (ms_step * 1e-3) / 1e6, 1)}))
    del ring, slab
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
