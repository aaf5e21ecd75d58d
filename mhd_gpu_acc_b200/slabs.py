"""One grid split into y-slabs: the multi-GPU decomposition of a single large
grid (one slab per GPU), and the same decomposition on one device.

A step of the split scheme needs, between its two sweeps, the two x-swept rows
on each side of a slab boundary: the y-sweep of row j reads rows j-2 .. j+2.
The x-sweep is row-local and the CFL maximum is a max over cells, so a step on
P slabs is
    M = the global CFL maximum of U              (a max over the slabs' clocks)
    ch = M; dt = cfl * min(dx, dy) / M           (identical on every slab)
    x-sweep of every slab, U -> T
    halo exchange: each slab's two first / last interior rows of T -> the
                   neighbour's ghost rows of T (2 x 9 rows per side)
    y-sweep of every slab, T -> U (two states per slab, as in mhd_run)
A side between two slabs is declared Dirichlet to the kernels: they then copy
(not compute) its ghost rows, which the exchange overwrites before the y-sweep
reads them, and no kernel reads a state's y-ghost rows otherwise.  The global
y boundaries keep their own type; with periodic y the slabs form a ring.

The step is device-resident: dt, c_h and the psi damping factor come from
each slab workspace's device clock (mhd_clock_start / mhd_sweep_clocked, as in
the single-grid graph loop mhd_run), the global CFL maximum is a max-reduce of
the clock slots between steps (int64 view of the bit pattern), and nothing is
read back to the host.  The y-sweep of each slab runs first over the interior
rows that need no halo (rows 2 .. n-3 of n), concurrently with the halo
exchange on a second stream, then over the two edge rows on each side once the
exchange has landed; the last edge launch gathers the Dirichlet ghost cells and
advances the clock.

`SlabGrid` keeps all slabs on the current device (one strided copy per halo
block through mhd_grid_copy_rows) and is bit-identical to the single-grid device loop
(mhd_run; every slab workspace steps with the global spacing,
mhd_set_spacing).  `DistSlabRun` holds one slab per rank; its exchange,
`exchange_rows`, sends the same rows with torch.distributed point-to-point
operations (NCCL on GPUs, gloo on CPU), and the CFL maximum is an
all-reduce(max) of the clock slot.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, load, mhd_grid, mhd_run_info
from .solver import F64, BoundaryConfig, BoundaryType, GpuWorkspace, Grid2DGPU, init_gpu_workspace

HALO = 2  # x-swept rows the y-sweep reads beyond a slab edge
EXCHANGED = int(BoundaryType.Dirichlet)  # kernel boundary type of a side filled by the exchange
SWEEP_NO_GATHER, SWEEP_NO_ADVANCE = 1, 2  # mhd_sweep_clocked flags


def y_windows(n: int, exchanged: bool) -> tuple[list[tuple[int, int, int]], list[tuple[int, int, int]]]:
    """(row0, nrows, flags) launches of a slab's y-sweep: those that read no halo
    row (run while the exchange proceeds) and those after it.  Exactly one launch
    gathers the Dirichlet ghost cells and advances the clock: the last one."""
    if not exchanged or n <= 2 * HALO:
        return [], [(0, 0, 0)]
    quiet = SWEEP_NO_GATHER | SWEEP_NO_ADVANCE
    return [(HALO, n - 2 * HALO, quiet)], [(0, HALO, quiet), (n - HALO, HALO, 0)]


class _DevicePtr:
    """__cuda_array_interface__ of a device pointer (shape, typestr)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def clock_slot(ws, parity: int):
    """int64 torch view of a workspace's device-clock slot (mhd_clock_slot)."""
    import torch

    p = C.c_void_p()
    check(load().mhd_clock_slot(ws.ptr, int(parity), C.byref(p)), "mhd_clock_slot")
    return torch.as_tensor(_DevicePtr(p.value, (1,), "<i8"), device="cuda")


def _sweep(ws, src, dst, solver, bc_arr, direction, parity, row0=0, nrows=0, flags=0):
    check(load().mhd_sweep_clocked(ws.ptr, C.byref(src.g), C.byref(dst.g), int(solver), bc_arr, direction, parity,
                                   row0, nrows, flags), "mhd_sweep_clocked")


def slab_rows(ny: int, parts: int) -> list[tuple[int, int]]:
    """Interior row ranges [r0, r1) of `parts` slabs, sizes differing by at most one."""
    if parts < 1 or parts > ny // HALO:
        raise ValueError(f"cannot split {ny} rows into {parts} slabs of >= {HALO} rows")
    base, extra = divmod(ny, parts)
    out, r0 = [], 0
    for p in range(parts):
        r1 = r0 + base + (1 if p < extra else 0)
        out.append((r0, r1))
        r0 = r1
    return out


def neighbours(p: int, parts: int, periodic_y: bool) -> tuple[int | None, int | None]:
    """(slab below, slab above) of slab p; None at a non-periodic global edge."""
    below = p - 1 if p > 0 else (parts - 1 if periodic_y and parts > 1 else None)
    above = p + 1 if p < parts - 1 else (0 if periodic_y and parts > 1 else None)
    return below, above


def slab_bc(bc, p: int, parts: int) -> tuple[int, int, int, int]:
    """Boundary types handed to the kernels for slab p: the global left/right, and
    the global bottom/top only on the outer slabs of a non-periodic y direction;
    sides that receive an exchange are Dirichlet (ghost rows copied, then overwritten)."""
    b = BoundaryConfig.of(bc)
    periodic_y = int(b.bottom) == 0 and int(b.top) == 0
    below, above = neighbours(p, parts, periodic_y)
    if parts == 1:
        return (int(b.left), int(b.right), int(b.bottom), int(b.top))
    return (int(b.left), int(b.right), EXCHANGED if below is not None else int(b.bottom),
            EXCHANGED if above is not None else int(b.top))


def slab_extent(y_min: float, y_max: float, ny: int, r0: int, r1: int) -> tuple[float, float]:
    """y extent of slab rows [r0, r1) of the global grid.  The slab's workspace
    is also given the global spacing (mhd_set_spacing), because
    (y1 - y0) / (r1 - r0) need not round back to the global dy."""
    dy = (y_max - y_min) / ny
    return y_min + r0 * dy, y_min + r1 * dy


def halo_copies(rows, ng: int, periodic_y: bool):
    """(src slab, src storage row, dst slab, dst storage row) of every 2-row block
    of the exchange: slab p's top interior rows go to the bottom ghost rows of the
    slab above, its bottom interior rows to the top ghost rows of the slab below."""
    parts = len(rows)
    out = []
    for p, (r0, r1) in enumerate(rows):
        n = r1 - r0
        below, above = neighbours(p, parts, periodic_y)
        if above is not None:
            out.append((p, ng + n - HALO, above, ng - HALO))
        if below is not None:
            nb = rows[below][1] - rows[below][0]
            out.append((p, ng, below, ng + nb))
    return out


class SlabGrid:
    """A grid of nx x ny cells held as `parts` y-slabs on the current device."""

    def __init__(self, nx: int, ny: int, ng: int, extent, parts: int, dtype: int = F64):
        self.nx, self.ny, self.ng, self.parts, self.dtype = nx, ny, ng, parts, dtype
        self.extent = tuple(float(v) for v in extent)
        x0, x1, y0, y1 = self.extent
        self.rows = slab_rows(ny, parts)
        self.U, self.T, self.ws = [], [], []
        for r0, r1 in self.rows:
            e = (x0, x1) + slab_extent(y0, y1, ny, r0, r1)
            U = Grid2DGPU(nx, r1 - r0, ng, *e, dtype)
            self.U.append(U)
            self.T.append(Grid2DGPU(nx, r1 - r0, ng, *e, dtype))
            ws = GpuWorkspace()
            init_gpu_workspace(ws, U)
            check(load().mhd_set_spacing(ws.ptr, (x1 - x0) / nx, (y1 - y0) / ny), "mhd_set_spacing")
            self.ws.append(ws)

    def upload(self, host: np.ndarray) -> None:
        """Global dense FP64 SoA (9, ny+2ng, nx+2ng) -> slabs (each with its ng ghost rows)."""
        ng = self.ng
        for (r0, r1), U, T in zip(self.rows, self.U, self.T):
            part = np.ascontiguousarray(host[:, r0:r1 + 2 * ng, :])
            for g in (U, T):
                g.upload(part)

    def download(self) -> np.ndarray:
        """Slabs -> global array; the global ghost rows come from the outer slabs."""
        ng = self.ng
        out = np.empty((9, self.ny + 2 * ng, self.nx + 2 * ng))
        for p, ((r0, r1), U) in enumerate(zip(self.rows, self.U)):
            a = U.download()
            lo = 0 if p == 0 else ng
            hi = (r1 - r0 + 2 * ng) if p == self.parts - 1 else (r1 - r0 + ng)
            out[:, r0 + lo:r0 + hi, :] = a[:, lo:hi, :]
        return out

    def configure(self, gamma: float, limiter: int, cr: float | None = None, ch: float = 0.0) -> None:
        lib = load()
        for ws in self.ws:
            check(lib.mhd_set_gamma(ws.ptr, float(gamma)), "mhd_set_gamma")
            check(lib.mhd_set_ch(ws.ptr, float(ch)), "mhd_set_ch")
            ws.set_limiter(limiter)
            if cr is not None:
                ws.set_cr(cr)

    def start(self, cfl: float, t_end: float) -> None:
        """Starts every slab's device clock on the current torch stream and sets
        clock slot 0 to the global CFL maximum."""
        import torch

        self.stream = torch.cuda.current_stream()
        self.xstream = torch.cuda.Stream()
        lib = load()
        for ws, U in zip(self.ws, self.U):
            ws.set_stream(self.stream.cuda_stream)
            check(lib.mhd_clock_start(ws.ptr, C.byref(U.g), float(cfl), float(t_end)), "mhd_clock_start")
        self.slots = [[clock_slot(ws, par) for ws in self.ws] for par in (0, 1)]
        self._reduce(0)
        self.k = 0

    def _reduce(self, parity: int) -> None:
        import torch

        m = torch.max(torch.cat(self.slots[parity]))
        for s in self.slots[parity]:
            s.copy_(m.view(1))

    def step(self, solver: int, bc) -> None:
        """One split step of the whole grid, enqueued on the stream start() saw;
        nothing is read back (info() reads the clock)."""
        import torch

        b = BoundaryConfig.of(bc)
        periodic_y = int(b.bottom) == 0 and int(b.top) == 0
        par = self.k & 1
        bcs = [(C.c_int * 4)(*slab_bc(b, p, self.parts)) for p in range(self.parts)]
        exchanged = self.parts > 1
        for p in range(self.parts):
            _sweep(self.ws[p], self.U[p], self.T[p], solver, bcs[p], 0, par)
        copies = halo_copies(self.rows, self.ng, periodic_y)
        if copies:
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.xstream.wait_event(ev)
            lib = load()
            for s, sr, d, dr in copies:
                check(lib.mhd_grid_copy_rows(C.byref(self.T[s].g), sr, C.byref(self.T[d].g), dr, HALO,
                                             C.c_void_p(self.xstream.cuda_stream)), "mhd_grid_copy_rows")
        plans = [y_windows(r1 - r0, exchanged) for r0, r1 in self.rows]
        for p, (early, _) in enumerate(plans):  # rows that read no halo row, during the exchange
            for row0, nrows, flags in early:
                _sweep(self.ws[p], self.T[p], self.U[p], solver, bcs[p], 1, par, row0, nrows, flags)
        if copies:
            self.stream.wait_stream(self.xstream)
        for p, (_, late) in enumerate(plans):
            for row0, nrows, flags in late:
                _sweep(self.ws[p], self.T[p], self.U[p], solver, bcs[p], 1, par, row0, nrows, flags)
        self._reduce(par ^ 1)
        self.k += 1

    def info(self) -> mhd_run_info:
        """The clock (every slab's is the same): t, steps, dt, c_h, status."""
        info = mhd_run_info()
        for ws in self.ws:
            check(load().mhd_clock_read(ws.ptr, C.byref(info)), "mhd_clock_read")
        return info

    def synchronize(self) -> None:
        lib = load()
        for ws in self.ws:
            check(lib.mhd_synchronize(ws.ptr), "mhd_synchronize")

    def destroy(self) -> None:
        for ws in self.ws:
            ws.destroy()
        self.ws = []


def exchange_rows(state, rows_here: int, ng: int, below: int | None, above: int | None, dist) -> None:
    """Rank-to-rank halo exchange on a torch tensor `state` of shape
    (9, rows_here + 2 ng, width) holding this rank's x-swept slab: sends the two
    first / last interior rows to the ranks below / above and receives their rows
    into the ghost rows, with torch.distributed point-to-point operations (the
    collective steps are the same on every rank).  below / above are ranks or None.
    Messages between two ranks match in posting order, so every rank posts
    "send up, send down" and then "receive from below, receive from above": with
    two ranks in a periodic ring (below == above) the first message is still the
    sender's top rows, and it lands in the receiver's bottom ghost rows."""
    import torch

    ops, recv = [], []
    if above is not None:
        ops.append(dist.P2POp(dist.isend, state[:, ng + rows_here - HALO:ng + rows_here, :].contiguous(), above))
    if below is not None:
        ops.append(dist.P2POp(dist.isend, state[:, ng:ng + HALO, :].contiguous(), below))
    if below is not None:
        buf = torch.empty_like(state[:, :HALO, :])
        ops.append(dist.P2POp(dist.irecv, buf, below))
        recv.append((buf, ng - HALO))
    if above is not None:
        buf = torch.empty_like(state[:, :HALO, :])
        ops.append(dist.P2POp(dist.irecv, buf, above))
        recv.append((buf, ng + rows_here))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for buf, r in recv:
        state[:, r:r + HALO, :] = buf


class _DeviceRows:
    """__cuda_array_interface__ view (9, ny + 2 ng, pitch) of a grid's device slab."""

    def __init__(self, g: mhd_grid):
        tny = g.ny + 2 * g.ng
        es = 8 if g.dtype == F64 else 4
        self.__cuda_array_interface__ = {
            "shape": (9, tny, int(g.pitch)), "typestr": "<f8" if es == 8 else "<f4",
            "strides": (int(g.plane) * es, int(g.pitch) * es, es), "data": (int(g.data), False), "version": 3,
        }


def grid_tensor(g: mhd_grid):
    """A torch tensor sharing the device memory of grid g (no copy)."""
    import torch

    return torch.as_tensor(_DeviceRows(g), device="cuda")


class DistSlabRun:
    """One slab per rank of a torch.distributed group (NCCL): the rank's rows of the
    global grid, its halo exchange with `exchange_rows` and the CFL maximum with an
    all-reduce(max).  Every rank calls step() the same number of times."""

    def __init__(self, nx: int, ny: int, ng: int, extent, dtype: int = F64):
        import torch.distributed as dist

        self.dist = dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.nx, self.ny, self.ng = nx, ny, ng
        self.extent = tuple(float(v) for v in extent)
        self.rows = slab_rows(ny, self.world)
        r0, r1 = self.rows[self.rank]
        x0, x1, y0, y1 = self.extent
        e = (x0, x1) + slab_extent(y0, y1, ny, r0, r1)
        self.U = Grid2DGPU(nx, r1 - r0, ng, *e, dtype)
        self.T = Grid2DGPU(nx, r1 - r0, ng, *e, dtype)
        self.ws = GpuWorkspace()
        init_gpu_workspace(self.ws, self.U)
        self.dx, self.dy = (x1 - x0) / nx, (y1 - y0) / ny
        check(load().mhd_set_spacing(self.ws.ptr, self.dx, self.dy), "mhd_set_spacing")

    def upload(self, host: np.ndarray) -> None:
        """This rank's rows (with ghost rows) of the global dense FP64 SoA array."""
        r0, r1 = self.rows[self.rank]
        part = np.ascontiguousarray(host[:, r0:r1 + 2 * self.ng, :])
        for g in (self.U, self.T):
            g.upload(part)

    def start(self, cfl: float, t_end: float) -> None:
        """Starts this rank's device clock on the current torch stream; clock slot 0
        becomes the global CFL maximum (all-reduce(max) across ranks)."""
        import torch

        self.stream = torch.cuda.current_stream()
        self.xstream = torch.cuda.Stream()
        self.ws.set_stream(self.stream.cuda_stream)
        check(load().mhd_clock_start(self.ws.ptr, C.byref(self.U.g), float(cfl), float(t_end)), "mhd_clock_start")
        self.slots = [clock_slot(self.ws, par) for par in (0, 1)]
        self.dist.all_reduce(self.slots[0], op=self.dist.ReduceOp.MAX)
        self.k = 0

    def step(self, solver: int, bc) -> None:
        """One split step of this rank's slab, enqueued without any host round trip:
        x-sweep; the halo exchange on a second stream while the y-sweep does the
        rows that need no halo; the edge rows; all-reduce(max) of the next CFL
        maximum.  Every rank calls it the same number of times."""
        import torch

        b = BoundaryConfig.of(bc)
        periodic_y = int(b.bottom) == 0 and int(b.top) == 0
        par = self.k & 1
        sbc = (C.c_int * 4)(*slab_bc(b, self.rank, self.world))
        _sweep(self.ws, self.U, self.T, solver, sbc, 0, par)
        below, above = neighbours(self.rank, self.world, periodic_y)
        r0, r1 = self.rows[self.rank]
        exchanged = below is not None or above is not None
        early, late = y_windows(r1 - r0, exchanged)
        if exchanged:
            ev = torch.cuda.Event()
            ev.record(self.stream)
            self.xstream.wait_event(ev)
            with torch.cuda.stream(self.xstream):
                exchange_rows(grid_tensor(self.T.g), r1 - r0, self.ng, below, above, self.dist)
        for row0, nrows, flags in early:
            _sweep(self.ws, self.T, self.U, solver, sbc, 1, par, row0, nrows, flags)
        if exchanged:
            self.stream.wait_stream(self.xstream)
        for row0, nrows, flags in late:
            _sweep(self.ws, self.T, self.U, solver, sbc, 1, par, row0, nrows, flags)
        self.dist.all_reduce(self.slots[par ^ 1], op=self.dist.ReduceOp.MAX)
        self.k += 1

    def info(self) -> mhd_run_info:
        info = mhd_run_info()
        check(load().mhd_clock_read(self.ws.ptr, C.byref(info)), "mhd_clock_read")
        return info

    def destroy(self) -> None:
        self.ws.destroy()
