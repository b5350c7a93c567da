"""Generate the golden fixtures by running the reference solver itself.

The reference's PyTorch modules are imported unmodified from a checkout of
yasahi-hpc/JAX-PyTorch-Vlasov (its root given by $VLASOV_REFERENCE) and
run eagerly on the CPU (TORCHDYNAMO_DISABLE=1). They
import xarray only for their netCDF writer, which is never called here, so
an empty stand-in module is registered first.

Inputs are regenerated from the seeds recorded in each fixture
(numpy.random.default_rng), so the files hold outputs only.

    VLASOV_REFERENCE=<checkout> python tests/golden/make_golden.py         # small cases + C1 history
    VLASOV_REFERENCE=<checkout> python tests/golden/make_golden.py --long  # also the C2 / C3 / 1D histories
"""
from __future__ import annotations

import argparse
import importlib.machinery
import importlib.util
import math
import os
import sys
import time
import types

os.environ.setdefault("TORCHDYNAMO_DISABLE", "1")

import numpy as np  # noqa: E402
import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("VLASOV_REFERENCE", "")
if not REF or not os.path.isdir(REF):
    sys.exit("make_golden.py: set VLASOV_REFERENCE to the root of a yasahi-hpc/JAX-PyTorch-Vlasov checkout")


def _load_reference():
    stub = types.ModuleType("xarray")
    stub.__spec__ = importlib.machinery.ModuleSpec("xarray", None)
    sys.modules.setdefault("xarray", stub)

    def load(rel, name):
        spec = importlib.util.spec_from_file_location(name, os.path.join(REF, rel))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
        return mod

    r2 = load("simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py", "ref_vlasov2d2v")
    r1 = load("simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py", "ref_vlasov1d1v")
    return r2, r1


R2, R1 = _load_reference()
TD = {"f64": torch.float64, "f32": torch.float32}

# small anisotropic 2D2V grid used by the kernel-level cases
SMALL = dict(Nx=8, Ny=6, Nvx=10, Nvy=12, Lx=2.0 * math.pi, Ly=3.0, Vx_max=4.0, Vy_max=5.0)
STEP = dict(Nx=8, Ny=8, Nvx=16, Nvy=12, Lx=4.0 * math.pi, Ly=4.0 * math.pi, Vx_max=6.0, Vy_max=5.0)


def rng_f(seed, shape, dtype):
    return torch.from_numpy(np.random.default_rng(seed).random(shape)).to(TD[dtype])


def grid2(p, dtype):
    return R2.Grid.create(**p, device="cpu", dtype=TD[dtype])


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **{k: (v.detach().cpu().numpy() if torch.is_tensor(v) else np.asarray(v))
                                 for k, v in arrays.items()})
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.1f} KiB)")


def shifts_from_blocks(blocks, n):
    s = np.zeros(n, dtype=np.int64)
    for a, b, sh in blocks:
        s[a:b] = sh
    return s


# --------------------------------------------------------------------------
def gen_tables():
    """precompute_x_drift tables (shift per velocity, weights) at the
    benchmark grids, FP32 and FP64 (vlasov2D2V.py:670-714)."""
    out = {}
    cases = [
        ("c1", 32, 6.0, 4 * math.pi / 32, 0.05),
        ("c2", 64, 8.0, 10 * math.pi / 64, 0.025),
        ("c3", 128, 6.0, 4 * math.pi / 128, 0.05),
        ("ref128", 128, 5.0, 4 * math.pi / 128, 0.025),
        ("oned4096", 4096, 5.0, 4 * math.pi / 4096, 0.025),
    ]
    for tag, n, vmax, dx, half_dt in cases:
        for dt in ("f32", "f64"):
            v = torch.linspace(-vmax, vmax, n, dtype=TD[dt])
            blocks, W = R2.precompute_x_drift(v, half_dt, dx, TD[dt])
            out[f"{tag}_{dt}_v"] = v
            out[f"{tag}_{dt}_shift"] = shifts_from_blocks(blocks, n)
            out[f"{tag}_{dt}_W"] = W
            out[f"{tag}_{dt}_meta"] = np.array([n, vmax, dx, half_dt])
    alpha = torch.from_numpy(np.random.default_rng(7).random(64))
    out["alpha"] = alpha
    out["lag5_f64"] = R2.lagrange5_weights(alpha)
    out["lag5_f32"] = R2.lagrange5_weights(alpha.float())
    save("tables", **out)


def gen_sweeps():
    """Single sweeps on the small grid: static drifts (advect_x_static),
    static kicks (advect_v_static, with and without window truncation),
    the gather sweep (advect_1d) and the roll/diag sweep (advect_1d_matrix_diag)."""
    out = {}
    for dt_name in ("f64", "f32"):
        g = grid2(SMALL, dt_name)
        f = rng_f(11, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt_name)
        dt = 0.1
        for axis in (0, 1):
            dx = g.dx if axis == 0 else g.dy
            vgrid = g.vx if axis == 0 else g.vy
            vmax = g.Vx_max if axis == 0 else g.Vy_max
            for fac in (0.3, 2.7, 6.0):
                v1 = vgrid / vmax * (fac * dx / dt)
                blocks, W = R2.precompute_x_drift(v1, dt, dx, TD[dt_name])
                o = R2.advect_x_static(f, W, blocks, g.stencil_offsets, axis)
                key = f"drift_{dt_name}_a{axis}_{fac}"
                out[key] = o
                out[key + "_v"] = v1
        for axis in (2, 3):
            dv = g.dvx if axis == 2 else g.dvy
            for fac in (0.3, 1.5, 4.2):
                E = (fac * dv / dt) * (
                    torch.sin(2.0 * torch.pi * torch.arange(g.Nx, dtype=TD[dt_name]) / g.Nx)[:, None]
                    * torch.cos(2.0 * torch.pi * torch.arange(g.Ny, dtype=TD[dt_name]) / g.Ny)[None, :]
                )
                S = int(np.ceil(float(E.abs().max()) * dt / dv)) + 1
                key = f"kick_{dt_name}_a{axis}_{fac}"
                out[key] = R2.advect_v_static(f, E, dt, dv, S, g.stencil_offsets, axis)
                out[key + "_E"] = E
                out[key + "_S"] = np.array(S)
                # window S=1 truncates taps once |E dt/dv| >= 1
                out[key + "_S1"] = R2.advect_v_static(f, E, dt, dv, 1, g.stencil_offsets, axis)
        # general gather sweep, per-line velocities as vlasov_step_impl builds them
        vel = {
            0: g.vx[None, :, None] * 1.7,
            1: g.vy[None, None, :] * -2.3,
            2: (torch.linspace(-3, 3, g.Nx * g.Ny, dtype=TD[dt_name]).reshape(g.Nx, g.Ny))[:, :, None],
            3: (torch.linspace(4, -4, g.Nx * g.Ny, dtype=TD[dt_name]).reshape(g.Nx, g.Ny))[:, :, None],
        }
        hx = {0: g.dx, 1: g.dy, 2: g.dvx, 3: g.dvy}
        idx = {0: g.x_indices, 1: g.y_indices, 2: g.vx_indices, 3: g.vy_indices}
        for axis in range(4):
            per = axis < 2
            out[f"gather_{dt_name}_a{axis}"] = R2.advect_1d(
                f, vel[axis], axis, dt, hx[axis], periodic=per,
                point_indices=idx[axis], stencil_offsets=g.stencil_offsets)
            out[f"diag_{dt_name}_a{axis}"] = R2.advect_1d_matrix_diag(
                f, vel[axis], axis, dt, hx[axis], periodic=per,
                point_indices=idx[axis], stencil_offsets=g.stencil_offsets)
        out[f"rho_{dt_name}"] = R2.compute_rho(f, g.dvx, g.dvy)
    out["seed"] = np.array(11)
    save("sweeps2d", **out)


def gen_poisson():
    """compute_poisson_real on seeded densities, even and odd sizes, plus
    the reference's analytic single-mode case (test_poisson.py)."""
    out = {}
    for (nx, ny) in ((16, 12), (15, 9), (9, 15), (8, 10)):
        for dt_name in ("f64", "f32"):
            p = dict(Nx=nx, Ny=ny, Nvx=4, Nvy=4, Lx=4.0 * math.pi, Ly=3.3, Vx_max=1.0, Vy_max=1.0)
            g = grid2(p, dt_name)
            rho = 1.0 + 0.01 * torch.from_numpy(np.random.default_rng(nx * 100 + ny).standard_normal((nx, ny)))
            rho = rho.to(TD[dt_name])
            Ex, Ey, drho, phi = R2.compute_poisson_real(rho, g.kx, g.ky, g.inv_ksq)
            key = f"p{nx}x{ny}_{dt_name}"
            out[key + "_Ex"], out[key + "_Ey"], out[key + "_drho"], out[key + "_phi"] = Ex, Ey, drho, phi
    save("poisson2d", **out)


def landau_ref(g, eps, k):
    x = g.x.to(torch.float64)
    y = g.y.to(torch.float64)
    vx = g.vx.to(torch.float64)
    vy = g.vy.to(torch.float64)
    sp = 1.0 + eps * (torch.cos(k * x)[:, None] + torch.cos(k * y)[None, :])
    fv = torch.exp(-0.5 * (vx[:, None] ** 2 + vy[None, :] ** 2)) / (2.0 * math.pi)
    return (sp[:, :, None, None] * fv[None, None]).to(g.x.dtype)


def two_stream_ref(g, eps, k, v0):
    x = g.x.to(torch.float64)
    y = g.y.to(torch.float64)
    vx = g.vx.to(torch.float64)
    vy = g.vy.to(torch.float64)
    M = lambda u: torch.exp(-0.5 * u * u) / math.sqrt(2.0 * math.pi)  # noqa: E731
    sp = 1.0 + eps * (torch.cos(k * x)[:, None] + torch.cos(k * y)[None, :])
    fv = (0.5 * (M(vx - v0) + M(vx + v0)))[:, None] * M(vy)[None, :]
    return (sp[:, :, None, None] * fv[None, None]).to(g.x.dtype)


def step_args(g, f0, dt, physics):
    return (f0, dt, g.x, g.y, g.vx, g.vy, g.kx, g.ky, g.inv_ksq,
            g.x_indices, g.y_indices, g.vx_indices, g.vy_indices, g.stencil_offsets,
            g.dx, g.dy, g.dvx, g.dvy, g.Nx, g.Ny, physics)


def gen_steps():
    """Three Strang steps of solvers 0/1/2 on a small Landau case, physics on and off."""
    out = {}
    g = grid2(STEP, "f64")
    f_init = landau_ref(g, 0.05, 0.5)
    f0 = torch.zeros(g.Nvx, g.Nvy, dtype=torch.float64)
    impl0 = getattr(R2.vlasov_step_impl, "_torchdynamo_orig_callable", R2.vlasov_step_impl)
    fns = {0: impl0, 1: R2.vlasov_step_matrix_diag, 2: R2.vlasov_step_gather_free}
    for phys in (True, False):
        for s, fn in fns.items():
            f = f_init
            for i in range(3):
                f, drho, phi = fn(f, *step_args(g, f0, 0.1, phys))
                key = f"s{s}_{'phys' if phys else 'free'}_n{i + 1}"
                out[key + "_drho"], out[key + "_phi"] = drho, phi
            out[f"s{s}_{'phys' if phys else 'free'}_f"] = f
    out["eps_k_dt"] = np.array([0.05, 0.5, 0.1])
    save("steps2d", **out)


def field_energy(g, drho):
    """W_E of the reference's own mid-step density, through its own Poisson."""
    Ex, Ey, _, _ = R2.compute_poisson_real(drho + 1.0, g.kx, g.ky, g.inv_ksq)
    Ex = Ex.to(torch.float64)
    Ey = Ey.to(torch.float64)
    return float(0.5 * torch.sum(Ex * Ex + Ey * Ey) * g.dx * g.dy), Ex, Ey


def gen_history(tag, p, dt, steps, ic, dtype="f64", snap_every=None):
    g = grid2(p, dtype)
    f = ic(g)
    f0 = torch.zeros(g.Nvx, g.Nvy, dtype=TD[dtype])
    blocks_x, W_x = R2.precompute_x_drift(g.vx, dt / 2.0, g.dx, TD[dtype])
    blocks_y, W_y = R2.precompute_x_drift(g.vy, dt / 2.0, g.dy, TD[dtype])
    offs = R2.static_stencil_offsets(g.stencil_offsets)
    we, mass, win = [], [], []
    snaps = {}
    t0 = time.time()
    for i in range(steps):
        f, drho, phi = R2.vlasov_step_gather_free_impl(
            f, dt, W_x, W_y, blocks_x, blocks_y, offs, g.kx, g.ky, g.inv_ksq,
            g.dvx, g.dvy, g.Nx, g.Ny, True, 1)
        w, Ex, Ey = field_energy(g, drho)
        we.append(w)
        mass.append(float(torch.sum(drho.to(torch.float64) + 1.0) * g.dx * g.dy))
        win.append(max(R2.check_v_window(Ex, dt, g.dvx, 1), R2.check_v_window(Ey, dt, g.dvy, 1)))
        if snap_every and (i + 1) % snap_every == 0:
            snaps[f"drho_{i + 1}"] = drho
        if (i + 1) % 10 == 0:
            print(f"  {tag} step {i + 1}/{steps} W_E={w:.6e} ({time.time() - t0:.0f}s)", flush=True)
    save(f"history_{tag}", W_E=np.array(we), mass=np.array(mass), kick_window=np.array(win),
         drho_final=drho, phi_final=phi, params=np.array([dt, steps]), **snaps)


# --------------------------------------------------------------------------
def gen_1d():
    out = {}
    for dt_name in ("f64", "f32"):
        g = R1.Grid.create(24, 20, 4.0 * math.pi, 5.0, device="cpu", dtype=TD[dt_name])
        f = rng_f(5, (24, 20), dt_name)
        dt = 0.1
        for fac in (0.4, 3.3):
            v1 = g.v / g.V_max * (fac * g.dx / dt)
            blocks, W = R1.precompute_x_drift(v1, dt, g.dx, TD[dt_name])
            out[f"drift_{dt_name}_{fac}"] = R1.advect_x_static(f, W, blocks, g.stencil_offsets)
            out[f"drift_{dt_name}_{fac}_v"] = v1
        for fac in (0.3, 2.2):
            E = (fac * g.dv / dt) * torch.sin(2 * torch.pi * torch.arange(24, dtype=TD[dt_name]) / 24)
            S = int(np.ceil(float(E.abs().max()) * dt / g.dv)) + 1
            out[f"kick_{dt_name}_{fac}"] = R1.advect_v_static(f, E, dt, g.dv, S, g.stencil_offsets)
            out[f"kick_{dt_name}_{fac}_E"] = E
        # gather sweeps: x on f.T with per-row velocities, v with E per row
        vx_rows = g.v * 1.3
        out[f"gx_{dt_name}"] = R1.advect_1d_vectorized(
            f.T, vx_rows, dt, g.x_indices, g.x_batch_offsets, g.stencil_offsets, g.dx, periodic=True).T
        Ev = torch.linspace(-2, 2, 24, dtype=TD[dt_name])
        out[f"gv_{dt_name}"] = R1.advect_1d_vectorized(
            f, Ev, dt, g.v_indices, g.v_batch_offsets, g.stencil_offsets, g.dv, periodic=False)
        # Poisson: both forms
        fl = (1.0 + 0.01 * torch.cos(2 * torch.pi / g.L * g.x))[:, None] * torch.exp(-0.5 * g.v ** 2)[None, :] / math.sqrt(2 * math.pi)
        fl = fl.to(TD[dt_name])
        E, rho, phi = R1.solve_poisson_real(fl, g.inv_kx, g.inv_kx_sq, g.dv)
        out[f"pois_{dt_name}_E"], out[f"pois_{dt_name}_rho"], out[f"pois_{dt_name}_phi"] = E, rho, phi
        # three solver-0 and solver-2 steps, Landau IC
        for s, fn in ((0, getattr(R1.vlasov_step, "_torchdynamo_orig_callable", R1.vlasov_step)),
                      (2, R1.vlasov_step_gather_free)):
            fs = fl
            for i in range(3):
                fs, rho, phi = fn(fs, dt, g.v, g.inv_kx, g.inv_kx_sq, g.x_indices, g.v_indices,
                                  g.x_batch_offsets, g.v_batch_offsets, g.stencil_offsets,
                                  g.dx, g.dv, g.V_max, True)
                out[f"s{s}_{dt_name}_n{i + 1}_rho"], out[f"s{s}_{dt_name}_n{i + 1}_phi"] = rho, phi
            out[f"s{s}_{dt_name}_f"] = fs
    save("oned", **out)


def gen_helpers():
    """The reference's smaller public helpers of both modules: block_roll,
    build_v_tap_weights, the batched 2D sweep advect_1d_vectorized, the
    per-row form advect_1d_matrix_diag_core and its roll / banded-weight
    helpers, on seeded inputs. Inputs are regenerated from the seeds."""
    out = {}
    for dt_name in ("f64", "f32"):
        T = TD[dt_name]
        g = grid2(SMALL, dt_name)
        f = rng_f(21, (g.Nx, g.Ny, g.Nvx, g.Nvy), dt_name)
        for axis, vel in ((0, g.vx), (1, g.vy)):
            h = g.dx if axis == 0 else g.dy
            blocks, _ = R2.precompute_x_drift(vel * 3.1, 0.1, h, T)
            out[f"broll_{dt_name}_a{axis}"] = R2.block_roll(f, blocks, axis, axis + 2)
        E = (0.7 * torch.sin(torch.arange(g.Nx * g.Ny, dtype=T).reshape(g.Nx, g.Ny))).to(T)
        for S in (1, 2):
            out[f"vtap_{dt_name}_S{S}"] = R2.build_v_tap_weights(E, 0.1, g.dvx, S, g.stencil_offsets)
        B, N = 7, 19
        fb = rng_f(22, (B, N), dt_name)
        vb = torch.linspace(-3.0, 4.0, B, dtype=T)
        ve = (2.5 * torch.cos(torch.arange(B * N, dtype=T) * 0.37).reshape(B, N)).to(T)
        for per in (True, False):
            tag = "p" if per else "d"
            out[f"avec_{dt_name}_rows_{tag}"] = R2.advect_1d_vectorized(fb, vb, 0.1, 0.25, periodic=per)
            out[f"avec_{dt_name}_elem_{tag}"] = R2.advect_1d_vectorized(fb, ve, 0.1, 0.25, periodic=per)
            out[f"mdcore_{dt_name}_{tag}"] = R2.advect_1d_matrix_diag_core(fb, vb, 0.1, 0.25, g.stencil_offsets,
                                                                          periodic=per)
        sh = torch.tensor([-3, 0, 2, 5, -7, 19, 40], dtype=torch.int64)
        out[f"rollb_{dt_name}"] = R2._roll_batch(fb, sh)
        al = torch.linspace(0.05, 0.95, B, dtype=T)
        out[f"dw_{dt_name}"] = R2.build_diag_weights(g.stencil_offsets, sh, al, N)
        # 1D1V forms
        g1 = R1.Grid.create(24, 20, 4.0 * math.pi, 5.0, device="cpu", dtype=T)
        f1 = rng_f(23, (24, 20), dt_name)
        blocks1, _ = R1.precompute_x_drift(g1.v * 2.3, 0.1, g1.dx, T)
        out[f"broll1_{dt_name}"] = R1.block_roll(f1, blocks1)
        E1 = (0.9 * torch.sin(torch.arange(24, dtype=T))).to(T)
        out[f"vtap1_{dt_name}"] = R1.build_v_tap_weights(E1, 0.1, g1.dv, 1, g1.stencil_offsets)
        shc = torch.arange(20, dtype=torch.int64) - 9
        shr = torch.arange(24, dtype=torch.int64) * 3 - 30
        out[f"rollc1_{dt_name}"] = R1._roll_columns(f1, shc)
        out[f"rollr1_{dt_name}"] = R1._roll_rows(f1, shr)
        al1 = torch.linspace(0.1, 0.9, 24, dtype=T)
        out[f"vdw1_{dt_name}"] = R1.build_v_diag_weights(g1.stencil_offsets, shr, al1, 20)
    save("helpers", **out)


def gen_history_1d(tag, nx, nv, L, vmax, eps, dt, steps):
    g = R1.Grid.create(nx, nv, L, vmax, device="cpu", dtype=torch.float64)
    f = (1.0 + eps * torch.cos(2 * math.pi / L * g.x))[:, None] * (
        torch.exp(-0.5 * g.v ** 2) / math.sqrt(2 * math.pi))[None, :]
    blocks, W = R1.precompute_x_drift(g.v, dt / 2.0, g.dx, torch.float64)
    offs = R1.static_stencil_offsets(g.stencil_offsets)
    rhos = []
    for i in range(steps):
        f, rho, phi = R1.vlasov_step_gather_free_impl(f, dt, W, blocks, offs, g.inv_kx, g.inv_kx_sq,
                                                      g.dv, True, 1)
        rhos.append(rho.numpy().copy())
    save(f"history_{tag}", rho=np.stack(rhos), phi_final=phi,
         params=np.array([nx, nv, L, vmax, eps, dt, steps]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--long", action="store_true")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    torch.set_num_threads(os.cpu_count() or 1)
    c1 = dict(Nx=32, Ny=32, Nvx=32, Nvy=32, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0)
    jobs = {
        "tables": gen_tables,
        "sweeps": gen_sweeps,
        "poisson": gen_poisson,
        "steps": gen_steps,
        "oned": gen_1d,
        "helpers": gen_helpers,
        "c1": lambda: gen_history("c1", c1, 0.1, 100, lambda g: landau_ref(g, 0.01, 0.5), snap_every=25),
        "oned_landau": lambda: gen_history_1d("oned_landau", 128, 128, 4 * math.pi, 6.0, 0.01, 0.1, 200),
    }
    long_jobs = {
        "c2": lambda: gen_history(
            "c2", dict(Nx=64, Ny=64, Nvx=64, Nvy=64, Lx=10 * math.pi, Ly=10 * math.pi, Vx_max=8.0, Vy_max=8.0),
            0.05, 400, lambda g: two_stream_ref(g, 0.001, 0.2, 2.4), snap_every=100),
        "c3": lambda: gen_history(
            "c3", dict(Nx=128, Ny=128, Nvx=128, Nvy=128, Lx=4 * math.pi, Ly=4 * math.pi, Vx_max=6.0, Vy_max=6.0),
            0.1, 20, lambda g: landau_ref(g, 0.05, 0.5), snap_every=10),
    }
    if a.long:
        jobs.update(long_jobs)
    only = set(filter(None, a.only.split(",")))
    for name, fn in {**jobs, **long_jobs}.items():
        if (only and name in only) or (not only and name in jobs):
            print(f"[{name}]", flush=True)
            fn()


if __name__ == "__main__":
    main()
