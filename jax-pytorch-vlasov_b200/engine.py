"""Stateful steppers: device tables, scratch and ping-pong buffers of one run,
one library call per Strang step, optional CUDA-graph capture of the loop.

Stepper2D / Stepper1D are what Vlasov.run and bench.py drive. The step is
the schedule of vlasov_step_gather_free_impl (vlasov2D2V.py:1043-1083,
vlasov1D1V.py:668-701) executed by vp_step2d / vp_step1d.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from . import ops


class _Stepper:
    """Shared run loop: eager steps, or chunks of `graph_chunk` steps captured
    once per (input buffer, output buffer) pair and replayed."""

    _lib_fn = ""

    def _init_common(self, dtype, device, physics_mode, window, diagnostics):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError(f"{type(self).__name__} runs on a CUDA device only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.physics_mode = bool(physics_mode)
        self.window = int(window)
        self.diagnostics = int(diagnostics)  # 0 none, 1 field energy + mass, 2 + L2 / kinetic moments
        self.diag = torch.zeros(L.DIAG_COUNT, dtype=torch.float64, device=self.device)
        # device status word the steps OR VP_STATUS_* bits into (read by check())
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.test_stall = 0  # test hook of vp_step2d (see vlasov_b200.h); 0 in normal use
        self._graphs = {}
        self._bufs = [None, None]

    def empty_f(self) -> torch.Tensor:
        return torch.empty(self.shape, dtype=self.dtype, device=self.device)

    def check(self) -> None:
        """Synchronise with the steps issued so far and raise VlasovError if
        one of them reported a device wait that ran out (its share of f was
        filled with NaN) or a non-finite field energy or mass; the status
        word is cleared either way."""
        bits = int(self.status.item())
        if bits:
            self.status.zero_()
            what = []
            if bits & L.STATUS_WAIT_TIMEOUT:
                what.append("a device wait ran out (the affected part of f is NaN)")
            if bits & L.STATUS_NONFINITE:
                what.append("non-finite field energy or mass")
            raise L.VlasovError(f"{type(self).__name__}: " + "; ".join(what or [f"status {bits:#x}"]))

    # ---- equilibrium split -------------------------------------------------
    def _set_equilibrium(self, factors, spacings):
        """factors: 1D equilibrium factors along each velocity dim (float64),
        or None. Sets the device copies and the equilibrium density."""
        if factors is None:
            self.eq = None
            self.eq_moment = 0.0
            return
        fs = [torch.as_tensor(f, dtype=torch.float64).detach().reshape(-1).cpu() for f in factors]
        self.eq = [f.to(self.device) for f in fs]
        m = 1.0
        for f, dv in zip(fs, spacings):
            m *= float(f.sum()) * dv
        self.eq_moment = m

    def feq(self) -> torch.Tensor:
        """The equilibrium over the velocity grid (float64), broadcastable to f."""
        if self.eq is None:
            raise ValueError("no equilibrium split configured")
        if len(self.eq) == 1:
            return self.eq[0][None, :]
        return (self.eq[0][:, None] * self.eq[1][None, :])[None, None]

    def split(self, f: torch.Tensor) -> torch.Tensor:
        """State g = f - feq in the storage dtype (f given as the full f)."""
        return (f.to(torch.float64) - self.feq()).to(self.dtype).contiguous()

    def join(self, g: torch.Tensor) -> torch.Tensor:
        """The full f = feq + g (float64)."""
        return g.to(torch.float64) + self.feq()

    def _check(self, f):
        if (tuple(f.shape) != self.shape or f.dtype != self.dtype or f.device != self.device
                or not f.is_contiguous()):
            raise ValueError(f"f must be a contiguous {self.dtype} tensor of shape {self.shape} on {self.device}")

    def _desc(self, f_in, f_out, diag):
        raise NotImplementedError

    def step(self, f_in: torch.Tensor, f_out: torch.Tensor | None = None, diag: torch.Tensor | None = None):
        """One Strang step f_in -> f_out (a new tensor if None). Mid-step
        fields land in the stepper's field buffers; diagnostics in `diag`
        (default self.diag) when enabled."""
        self._check(f_in)
        f_out = self.empty_f() if f_out is None else f_out
        self._check(f_out)
        if diag is None and self.diagnostics:
            diag = self.diag
        desc = self._desc(f_in, f_out, diag)
        L.call(self._lib_fn, ctypes.byref(desc), ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
        return f_out

    def _partner(self, f):
        """A persistent second buffer distinct from f (and from f_tmp)."""
        if self._bufs[0] is None:
            self._bufs[0] = self.empty_f()
        if f.data_ptr() == self._bufs[0].data_ptr():
            if self._bufs[1] is None:
                self._bufs[1] = self.empty_f()
            return self._bufs[1]
        return self._bufs[0]

    def run(self, f: torch.Tensor, nsteps: int, history: torch.Tensor | None = None, graph: bool = False,
            graph_chunk: int = 10) -> torch.Tensor:
        """Advance f by nsteps and return the buffer holding the result (f
        itself after an even number of steps). history: optional float64
        [nsteps, VP_DIAG_COUNT] per-step diagnostics."""
        self._check(f)
        a, b = f, self._partner(f)
        done = 0
        if graph:
            k = max(2, graph_chunk + (graph_chunk & 1))  # even: every replay returns to `a`
            while nsteps - done >= k:
                key = (a.data_ptr(), b.data_ptr(), k)
                entry = self._graphs.get(key)
                if entry is None:
                    stage = torch.zeros((k, L.DIAG_COUNT), dtype=torch.float64, device=self.device)
                    s = torch.cuda.Stream(self.device)
                    s.wait_stream(torch.cuda.current_stream(self.device))
                    with torch.cuda.stream(s):  # first launches outside the capture
                        self.step(a, b, stage[0])
                        self.step(b, a, stage[1])
                    torch.cuda.current_stream(self.device).wait_stream(s)
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        x, y = a, b
                        for i in range(k):
                            self.step(x, y, stage[i])
                            x, y = y, x
                    self._graphs[key] = (g, stage)
                    if history is not None:
                        history[done: done + 2].copy_(stage[:2])
                    done += 2  # the two launches before the capture advanced the state
                    continue
                g, stage = entry
                g.replay()
                if history is not None:
                    history[done: done + k].copy_(stage)
                done += k
        for i in range(done, nsteps):
            self.step(a, b, history[i] if history is not None else None)
            a, b = b, a
        return a


class Stepper2D(_Stepper):
    """One 2D2V configuration: grid sizes, extents, dt and storage dtype.

    The velocity grids are built as Grid.create builds them
    (vlasov2D2V.py:146-156: linspace(-V, V, N) in the run precision, dv =
    2V/(N-1)), unless vx / vy are given. Drift tables are computed in the
    storage dtype's precision exactly as precompute_x_drift does.
    window: kick window S (-1: exact kick for any |E dt/dv|; the reference
    solver 2 uses S = 1, which equals the exact kick while |E dt/dv| < 1).
    diagnostics: 0 none, 1 field energy / mass / max shift, 2 also the L2 and
    kinetic moments after the kicks.
    """

    _lib_fn = "vp_step2d"

    def __init__(self, Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt, dtype=torch.float32, device="cuda",
                 physics_mode=True, window=-1, diagnostics=1, vx=None, vy=None, equilibrium=None,
                 precise_tables=False, fuse_drifts=True):
        self._init_common(dtype, device, physics_mode, window, diagnostics)
        self.shape = (int(Nx), int(Ny), int(Nvx), int(Nvy))
        # False: one sweep per axis even where the fused (x, y) plane passes
        # apply (same f; the density keeps the single-axis summation order)
        self.fuse_drifts = bool(fuse_drifts)
        self.Lx, self.Ly = float(Lx), float(Ly)
        self.dx, self.dy = self.Lx / Nx, self.Ly / Ny
        grid_dt = torch.float64 if (dtype == torch.float64 or precise_tables) else torch.float32
        vx_t = (torch.linspace(-Vx_max, Vx_max, Nvx, dtype=grid_dt) if vx is None
                else torch.as_tensor(vx).detach().cpu())
        vy_t = (torch.linspace(-Vy_max, Vy_max, Nvy, dtype=grid_dt) if vy is None
                else torch.as_tensor(vy).detach().cpu())
        self.dt = float(dt)
        self.dvx, self.dvy = 2 * Vx_max / (Nvx - 1), 2 * Vy_max / (Nvy - 1)
        self.tx = ops.DriftTable.from_velocity(vx_t, self.dt / 2.0, self.dx, dtype, self.device, precise_tables)
        self.ty = ops.DriftTable.from_velocity(vy_t, self.dt / 2.0, self.dy, dtype, self.device, precise_tables)
        self.kx, self.ky, self.inv_ksq = ops.spectral_2d(Nx, Ny, self.Lx, self.Ly, self.device)
        self.vx64 = vx_t.to(torch.float64).to(self.device)
        self.vy64 = vy_t.to(torch.float64).to(self.device)
        nb = L.query("vp_step2d_workspace_bytes", *self.shape)
        self.ws = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self.f_tmp = self.empty_f()
        z = lambda: torch.zeros((Nx, Ny), dtype=torch.float64, device=self.device)  # noqa: E731
        self.drho, self.phi, self.ex, self.ey = z(), z(), z(), z()
        if isinstance(equilibrium, str):
            if equilibrium != "maxwellian":
                raise ValueError("equilibrium: 'maxwellian', (A(vx), B(vy)) or None")
            m = lambda v: torch.exp(-0.5 * v.double() ** 2) / (2.0 * torch.pi) ** 0.5  # noqa: E731
            equilibrium = (m(vx_t), m(vy_t))
        # split storage f = A(vx) B(vy) + g: the state buffers hold g
        self._set_equilibrium(equilibrium, (self.dvx, self.dvy))

    def passes(self, f_in: torch.Tensor, f_out: torch.Tensor) -> tuple[int, bool]:
        """How step(f_in, f_out) runs: (passes over f, whether the position
        drifts go in pairs through the fused (x, y) plane passes)."""
        self._check(f_in)
        self._check(f_out)
        d = self._desc(f_in, f_out, None)
        flag = ctypes.c_int32(0)
        n = L.load().vp_step2d_passes(ctypes.byref(d), ctypes.byref(flag))
        if n < 0:
            raise L.VlasovError("vp_step2d_passes: " + L.load().vp_last_error().decode(errors="replace"))
        return int(n), bool(flag.value)

    def _desc(self, f_in, f_out, diag) -> L.Step2dDesc:
        d = L.Step2dDesc()
        d.dtype = L.dtype_code(self.dtype)
        d.nx, d.ny, d.nvx, d.nvy = self.shape
        d.dt, d.dx, d.dy, d.dvx, d.dvy = self.dt, self.dx, self.dy, self.dvx, self.dvy
        d.physics_mode = 1 if self.physics_mode else 0
        d.window = self.window
        d.diagnostics = self.diagnostics if diag is not None else 0
        d.shift_spread_x, d.shift_spread_y = self.tx.spread, self.ty.spread
        d.f_in, d.f_out, d.f_tmp = f_in.data_ptr(), f_out.data_ptr(), self.f_tmp.data_ptr()
        d.shift_x, d.W_x = self.tx.shift.data_ptr(), self.tx.W.data_ptr()
        d.shift_y, d.W_y = self.ty.shift.data_ptr(), self.ty.W.data_ptr()
        d.kx, d.ky, d.inv_ksq = self.kx.data_ptr(), self.ky.data_ptr(), self.inv_ksq.data_ptr()
        d.vx, d.vy = self.vx64.data_ptr(), self.vy64.data_ptr()
        d.drho, d.phi, d.ex, d.ey = (self.drho.data_ptr(), self.phi.data_ptr(), self.ex.data_ptr(),
                                     self.ey.data_ptr())
        d.diag = diag.data_ptr() if diag is not None else None
        d.workspace, d.workspace_bytes = self.ws.data_ptr(), self.ws.numel()
        if self.eq is not None:
            d.eq_vx, d.eq_vy = self.eq[0].data_ptr(), self.eq[1].data_ptr()
            d.eq_moment = self.eq_moment
        d.sweeps_only = 0 if getattr(self, "fuse_drifts", True) else 1
        d.status = self.status.data_ptr()
        d.test_stall = int(self.test_stall)
        return d


class Stepper1D(_Stepper):
    """One 1D1V configuration (f is (Nx, Nv), v contiguous); grids as
    Grid.create builds them (vlasov1D1V.py:95-122)."""

    _lib_fn = "vp_step1d"

    def __init__(self, Nx, Nv, L_, V_max, dt, dtype=torch.float32, device="cuda", physics_mode=True, window=-1,
                 diagnostics=1, v=None, equilibrium=None, precise_tables=False):
        self._init_common(dtype, device, physics_mode, window, diagnostics)
        self.shape = (int(Nx), int(Nv))
        self.L = float(L_)
        self.dx = self.L / Nx
        grid_dt = torch.float64 if (dtype == torch.float64 or precise_tables) else torch.float32
        v_t = torch.linspace(-V_max, V_max, Nv, dtype=grid_dt) if v is None else torch.as_tensor(v).detach().cpu()
        self.dv = 2 * V_max / (Nv - 1)
        self.dt = float(dt)
        self.table = ops.DriftTable.from_velocity(v_t, self.dt / 2.0, self.dx, dtype, self.device, precise_tables)
        self.inv_kx, self.inv_kx_sq = ops.spectral_1d(Nx, self.L, self.device)
        self.v64 = v_t.to(torch.float64).to(self.device)
        nb = L.query("vp_step1d_workspace_bytes", *self.shape)
        self.ws = torch.empty(nb, dtype=torch.uint8, device=self.device)
        self.f_tmp = self.empty_f()
        self.rho = torch.zeros(Nx, dtype=torch.float64, device=self.device)
        self.phi = torch.zeros_like(self.rho)
        self.e = torch.zeros_like(self.rho)
        if isinstance(equilibrium, str):
            if equilibrium != "maxwellian":
                raise ValueError("equilibrium: 'maxwellian', F(v) or None")
            equilibrium = torch.exp(-0.5 * v_t.double() ** 2) / (2.0 * torch.pi) ** 0.5
        self._set_equilibrium(None if equilibrium is None else (equilibrium,), (self.dv,))

    def _desc(self, f_in, f_out, diag) -> L.Step1dDesc:
        d = L.Step1dDesc()
        d.dtype = L.dtype_code(self.dtype)
        d.nx, d.nv = self.shape
        d.dt, d.dx, d.dv = self.dt, self.dx, self.dv
        d.physics_mode = 1 if self.physics_mode else 0
        d.window = self.window
        d.diagnostics = self.diagnostics if diag is not None else 0
        d.shift_spread = self.table.spread
        d.f_in, d.f_out, d.f_tmp = f_in.data_ptr(), f_out.data_ptr(), self.f_tmp.data_ptr()
        d.shift, d.W = self.table.shift.data_ptr(), self.table.W.data_ptr()
        d.inv_kx, d.inv_kx_sq, d.v = self.inv_kx.data_ptr(), self.inv_kx_sq.data_ptr(), self.v64.data_ptr()
        d.rho, d.phi, d.e = self.rho.data_ptr(), self.phi.data_ptr(), self.e.data_ptr()
        d.diag = diag.data_ptr() if diag is not None else None
        d.workspace, d.workspace_bytes = self.ws.data_ptr(), self.ws.numel()
        if self.eq is not None:
            d.eq_v = self.eq[0].data_ptr()
            d.eq_moment = self.eq_moment
        d.status = self.status.data_ptr()
        return d


class BatchStepper2D:
    """Independent 2D2V runs of uneven sizes and parameters advanced in
    lockstep: vp_batch2d_step launches one kernel per substep for all runs
    (at most 14 launches per step for up to 64 runs) and the state of run
    r is advanced in place in self.f[r]. Each run's step is vp_step2d's: the
    runs in `fused` (FP32, 32 <= Ny <= 64 a multiple of 8, Nvy a multiple of
    16, Nvx * Nvy of 32) take their drift pairs as fused passes, bit-identical to a Stepper2D
    with the fused passes; the others one sweep per axis (fuse_drifts=False:
    all of them).

    runs: sequence of dicts with Nx, Ny, Nvx, Nvy, Lx, Ly, Vx_max, Vy_max, dt
    (other keys are ignored). tiles: None (defaults), "auto" (the autotuner's
    cached choices, see autotune.py), or a dict with 3-tuples "block",
    "ctas_per_sm", "segments" per sweep kind (x drifts, y drifts, kick) and
    optionally "run_segments": one (x, y) pair per run.
    diagnostics 1: field energy, mass and max shift of every run per step.
    """

    def __init__(self, runs, dtype=torch.float32, device="cuda", physics_mode=True, window=-1, diagnostics=1,
                 tiles=None, precise_tables=False, graph_slots=10, fuse_drifts=True):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("BatchStepper2D runs on a CUDA device only")
        self.fuse_drifts = bool(fuse_drifts)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.dtype = dtype
        self.physics_mode = bool(physics_mode)
        self.diagnostics = int(diagnostics)
        self.window = int(window)
        self.params = [dict(r) for r in runs]
        n = len(self.params)
        if n == 0:
            raise ValueError("no runs")
        self.n_runs = n
        esz = torch.empty((), dtype=dtype).element_size()
        al = lambda b: (b + 255) // 256 * 256  # noqa: E731
        self.shapes, offs, wsoffs = [], [], []
        fbytes = wsbytes = 0
        for p in self.params:
            shape = (int(p["Nx"]), int(p["Ny"]), int(p["Nvx"]), int(p["Nvy"]))
            self.shapes.append(shape)
        # the rule of vp_batch2d_plan (the arenas keep every buffer 256-byte aligned)
        self.fused = [self.fuse_drifts and dtype == torch.float32 and 32 <= s[1] <= 64 and s[1] % 8 == 0
                      and s[3] % 16 == 0 and (s[2] * s[3]) % 32 == 0 for s in self.shapes]
        for p, shape in zip(self.params, self.shapes):
            offs.append(fbytes)
            fbytes += al(esz * shape[0] * shape[1] * shape[2] * shape[3])
            wsoffs.append(wsbytes)
            wsbytes += al(L.query("vp_step2d_workspace_bytes", *shape))
        # three arenas (state, two scratch) holding every run at 256-byte offsets
        self._arenas = [torch.empty(fbytes, dtype=torch.uint8, device=self.device) for _ in range(3)]
        self._ws = torch.empty(max(wsbytes, 256), dtype=torch.uint8, device=self.device)

        def view(arena, off, shape):
            nb = esz * shape[0] * shape[1] * shape[2] * shape[3]
            return arena[off: off + nb].view(dtype).view(shape)

        self.f = [view(self._arenas[0], o, s) for o, s in zip(offs, self.shapes)]
        self._s1 = [view(self._arenas[1], o, s) for o, s in zip(offs, self.shapes)]
        self._s2 = [view(self._arenas[2], o, s) for o, s in zip(offs, self.shapes)]
        self.slots = max(1, int(graph_slots))
        self.stage = torch.zeros((self.slots, n, L.DIAG_COUNT), dtype=torch.float64, device=self.device)
        # per-run device status words the steps OR VP_STATUS_* bits into (read by check())
        self.status = torch.zeros(n, dtype=torch.int32, device=self.device)
        self.drho, self.phi, self.tables = [], [], []
        runs_c = (L.BatchRun * n)()
        for r, (p, shape) in enumerate(zip(self.params, self.shapes)):
            Nx, Ny, Nvx, Nvy = shape
            Lx, Ly, dt = float(p["Lx"]), float(p["Ly"]), float(p["dt"])
            dx, dy = Lx / Nx, Ly / Ny
            dvx, dvy = 2 * p["Vx_max"] / (Nvx - 1), 2 * p["Vy_max"] / (Nvy - 1)
            grid_dt = torch.float64 if (dtype == torch.float64 or precise_tables) else torch.float32
            vx_t = torch.linspace(-p["Vx_max"], p["Vx_max"], Nvx, dtype=grid_dt)
            vy_t = torch.linspace(-p["Vy_max"], p["Vy_max"], Nvy, dtype=grid_dt)
            tx = ops.DriftTable.from_velocity(vx_t, dt / 2.0, dx, dtype, self.device, precise_tables)
            ty = ops.DriftTable.from_velocity(vy_t, dt / 2.0, dy, dtype, self.device, precise_tables)
            kx, ky, inv_ksq = ops.spectral_2d(Nx, Ny, Lx, Ly, self.device)
            drho = torch.zeros((Nx, Ny), dtype=torch.float64, device=self.device)
            phi = torch.zeros_like(drho)
            self.tables.append((tx, ty, kx, ky, inv_ksq))
            self.drho.append(drho)
            self.phi.append(phi)
            c = runs_c[r]
            c.nx, c.ny, c.nvx, c.nvy = Nx, Ny, Nvx, Nvy
            c.dt, c.dx, c.dy, c.dvx, c.dvy = dt, dx, dy, dvx, dvy
            c.window, c.shift_spread_x, c.shift_spread_y = self.window, tx.spread, ty.spread
            c.f, c.s1, c.s2 = self.f[r].data_ptr(), self._s1[r].data_ptr(), self._s2[r].data_ptr()
            c.shift_x, c.W_x = tx.shift.data_ptr(), tx.W.data_ptr()
            c.shift_y, c.W_y = ty.shift.data_ptr(), ty.W.data_ptr()
            c.kx, c.ky, c.inv_ksq = kx.data_ptr(), ky.data_ptr(), inv_ksq.data_ptr()
            c.drho, c.phi = drho.data_ptr(), phi.data_ptr()
            c.diag = self.stage[0, r].data_ptr()
            c.diag_slot_stride = n * L.DIAG_COUNT
            c.workspace = self._ws.data_ptr() + wsoffs[r]
            c.workspace_bytes = L.query("vp_step2d_workspace_bytes", *shape)
            c.status = self.status[r].data_ptr()
        self.dx = [c.dx for c in runs_c]
        self.dy = [c.dy for c in runs_c]
        self.dvx = [c.dvx for c in runs_c]
        self.dvy = [c.dvy for c in runs_c]
        self._runs_c = runs_c
        self._table_dev = None
        if isinstance(tiles, str):
            if tiles != "auto":
                raise ValueError("tiles: None, 'auto' or a dict")
            from . import autotune

            tiles = autotune.cached_tiles(self.shapes, dtype)
        self.retile(tiles)

    def retile(self, tiles=None):
        """Re-plan the batch with other tile shapes (drops captured graphs)."""
        n = self.n_runs
        t = None
        seg = (tiles or {}).get("run_segments")
        for r in range(n):
            sx, sy = (seg[r] if seg is not None else (0, 0))
            self._runs_c[r].segments_x, self._runs_c[r].segments_y = int(sx), int(sy)
        if tiles is not None or not self.fuse_drifts:
            t = L.BatchTiles()
            for key in ("block", "ctas_per_sm", "segments"):
                vals = (tiles or {}).get(key, (0, 0, 0))
                for i in range(L.BATCH_KINDS):
                    getattr(t, key)[i] = int(vals[i])
            t.sweeps_only = 0 if self.fuse_drifts else 1
        nb = L.query("vp_batch2d_table_bytes", n)
        table = ctypes.create_string_buffer(nb)
        L.call("vp_batch2d_plan", L.dtype_code(self.dtype), 1 if self.physics_mode else 0, self.diagnostics,
               self._runs_c, n, ctypes.byref(t) if t is not None else None, table, nb)
        host = torch.frombuffer(bytearray(table.raw), dtype=torch.uint8)
        if self._table_dev is not None:
            torch.cuda.current_stream(self.device).synchronize()  # no step may still read the old table
        self._table_host = table
        self._table_dev = host.to(self.device)
        self.tiles = tiles
        self._graphs = {}

    def check(self) -> None:
        """Synchronise with the steps issued so far and raise VlasovError if
        a run reported a device wait that ran out (a fused pass's CTA filled
        its share of f with NaN, on every run it served) or non-finite
        diagnostics; the status words are cleared either way."""
        bits = self.status.cpu()
        if bool(bits.any()):
            self.status.zero_()
            wait = [r for r in range(self.n_runs) if int(bits[r]) & L.STATUS_WAIT_TIMEOUT]
            bad = [r for r in range(self.n_runs) if int(bits[r]) & L.STATUS_NONFINITE]
            what = []
            if wait:
                what.append(f"a device wait ran out on runs {wait} (the affected parts of f are NaN)")
            if bad:
                what.append(f"non-finite field energy or mass on runs {bad}")
            raise L.VlasovError("BatchStepper2D: " + "; ".join(what))

    def set_test_stall(self, r: int, on: bool = True) -> None:
        """Test hook: make the first TMA wait of each CTA of the fused passes
        that starts on run r run out (1 s bound) in the following steps; re-plans
        the batch."""
        self._runs_c[r].test_stall = 1 if on else 0
        self.retile(self.tiles)

    def phase_ms(self, steps: int = 3):
        """Mean per-substep device times (ms) of `steps` eager steps, keyed by
        the phase names of the step (drift_x1, drift_y1_rho, field, kick,
        drift_y2, drift_x2, diag). The state advances."""
        nph = 7
        rows = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * nph)] for _ in range(steps)]
        for row in rows:
            for e in row:
                e.record()
        torch.cuda.synchronize(self.device)
        for row in rows:
            arr = (ctypes.c_void_p * (2 * nph))(*[e.cuda_event for e in row])
            self.step(0, events=arr)
        torch.cuda.synchronize(self.device)
        names = ("drift_x1", "drift_y1_rho", "field", "kick", "drift_y2", "drift_x2", "diag")
        return {nm: sum(row[2 * j].elapsed_time(row[2 * j + 1]) for row in rows) / steps
                for j, nm in enumerate(names)}

    @property
    def cells(self) -> int:
        return int(sum(s[0] * s[1] * s[2] * s[3] for s in self.shapes))

    def set_state(self, r: int, f: torch.Tensor):
        self.f[r].copy_(f.to(self.dtype))

    def step(self, slot: int = 0, events=None):
        """One Strang step of every run; diagnostics into self.stage[slot].
        events: optional ctypes array of 2*VP_PHASE_COUNT cudaEvent_t handles
        recorded around the substeps."""
        if not 0 <= slot < self.slots:
            raise ValueError(f"slot must be in [0, {self.slots})")
        L.call("vp_batch2d_step", self._table_host, ctypes.c_void_p(self._table_dev.data_ptr()), int(slot),
               ctypes.cast(events, ctypes.c_void_p) if events is not None else None,
               ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))

    def run(self, nsteps: int, history: torch.Tensor | None = None, graph: bool = True):
        """Advance every run by nsteps. history: optional float64
        [nsteps, n_runs, VP_DIAG_COUNT]. With graph=True, chunks of `slots`
        steps are captured once and replayed."""
        done = 0
        k = self.slots
        if graph and nsteps >= k:
            g = self._graphs.get(k)
            if g is None:
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                with torch.cuda.stream(s):  # the first launches outside the capture
                    self.step(0)
                torch.cuda.current_stream(self.device).wait_stream(s)
                if history is not None:
                    history[0].copy_(self.stage[0])
                done = 1
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    for i in range(k):
                        self.step(i)
                self._graphs[k] = g
            while nsteps - done >= k:
                g.replay()
                if history is not None:
                    history[done: done + k].copy_(self.stage)
                done += k
        while done < nsteps:
            self.step(0)
            if history is not None:
                history[done].copy_(self.stage[0])
            done += 1
