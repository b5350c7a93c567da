"""The C ABI library loads without a GPU, exports every entry point that
include/vlasov_b200.h declares, and the ctypes mirrors of its descriptor
structs have the C layout. Argument errors are reported before any CUDA call,
so they are checked here on the CPU."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "vlasov_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(vp_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def lib(vp):
    vp.build.build()
    return vp.load()


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("vp_drift", "vp_drift_rho", "vp_kick", "vp_kick2d", "vp_advect_gather", "vp_rho", "vp_poisson2d",
              "vp_poisson1d", "vp_step2d", "vp_step1d"):
        assert n in names


def test_every_declared_symbol_is_exported(lib, vp):
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in vlasov_b200.h but not exported"
        assert name in vp._lib.SIGNATURES, f"{name} has no ctypes signature"


def test_descriptor_layout_matches_c(vp, tmp_path):
    fields = {"vp_step2d_desc": vp._lib.Step2dDesc, "vp_step1d_desc": vp._lib.Step1dDesc,
              "vp_batch2d_run": vp._lib.BatchRun, "vp_batch_tiles": vp._lib.BatchTiles}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, cls in fields.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            a, b, v = ln.split()
            got[(a, b)] = int(v)
    for cname, cls in fields.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(cls)
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_argument_errors_without_gpu(lib, vp):
    L = vp._lib
    # null pointers and aliasing are rejected before any CUDA call
    rc = lib.vp_drift(None, None, L.VP_F32, 1, 8, 8, 1, 8, None, -1, None, None)
    assert rc == 1 and b"null" in lib.vp_last_error()
    p = ctypes.c_void_p(0x1000)
    rc = lib.vp_drift(p, p, L.VP_F32, 1, 8, 8, 1, 8, p, -1, p, None)
    assert rc == 1 and b"alias" in lib.vp_last_error()
    rc = lib.vp_drift(p, ctypes.c_void_p(0x2000), 7, 1, 8, 8, 1, 8, p, -1, p, None)
    assert rc == 2
    rc = lib.vp_kick(p, ctypes.c_void_p(0x2000), L.VP_F32, 4, 8, 1, p, L.VP_F64, 1, 0.1, 0.0, -1, None)
    assert rc == 1 and b"dv" in lib.vp_last_error()
    d = L.Step2dDesc()
    d.dtype, d.nx, d.ny, d.nvx, d.nvy = L.VP_F32, 8, 8, 8, 8
    d.f_in, d.f_out, d.f_tmp = 0x1000, 0x2000, 0x3000
    d.shift_x = d.W_x = d.shift_y = d.W_y = d.kx = d.ky = d.inv_ksq = 0x4000
    d.dvx = d.dvy = 1.0
    d.physics_mode = 1
    d.workspace, d.workspace_bytes = 0x5000, 16
    assert lib.vp_step2d(ctypes.byref(d), None) == 3  # workspace too small
    d.f_out = 0x1000
    assert lib.vp_step2d(ctypes.byref(d), None) == 1  # aliasing buffers
    assert lib.vp_step2d_workspace_bytes(128, 128, 128, 128) > 128 * 128 * 8
    # a field solve whose column transform would not fit a block's shared memory
    d.f_out = 0x2000
    d.nx = 2048
    assert lib.vp_step2d(ctypes.byref(d), None) == 5 and b"shared memory" in lib.vp_last_error()
    q = ctypes.c_void_p(0x6000)
    rc = lib.vp_poisson2d(q, 2048, 16, q, q, q, 0.1, 0.1, q, q, None, None, None, q, 1 << 30, None)
    assert rc == 5 and b"shared memory" in lib.vp_last_error()
    rc = lib.vp_poisson2d(q, 16, 4096, q, q, q, 0.1, 0.1, q, q, None, None, None, q, 1 << 30, None)
    assert rc == 5  # the inverse rows' shared memory: ny above about 3600
    rc = lib.vp_poisson2d(q, 1024, 2048, q, q, q, 0.1, 0.1, q, q, None, None, None, q, 16, None)
    assert rc == 3  # within the limits: the (too small) workspace is what fails


def _fake_run(L, lib, k, nx=16, ny=16, nvx=32, nvy=32):
    r = L.BatchRun()
    r.nx, r.ny, r.nvx, r.nvy = nx, ny, nvx, nvy
    r.dt, r.dx, r.dy, r.dvx, r.dvy = 0.05, 0.1, 0.1, 0.2, 0.2
    r.window, r.shift_spread_x, r.shift_spread_y = -1, 1, 1
    base = 0x10000000 * (k + 1)
    r.f, r.s1, r.s2 = base, base + 0x1000000, base + 0x2000000
    r.shift_x = r.W_x = r.shift_y = r.W_y = r.kx = r.ky = r.inv_ksq = base + 0x3000000
    r.workspace = base + 0x4000000
    r.workspace_bytes = lib.vp_step2d_workspace_bytes(nx, ny, nvx, nvy)
    return r


def test_batch_plan_on_host(lib, vp):
    """The batch plan is pure host work: it validates every run and fills the
    table without touching a device."""
    L = vp._lib
    runs = (L.BatchRun * 3)(*[_fake_run(L, lib, k, 16 + 8 * k, 16, 32 + 16 * (k % 2), 32) for k in range(3)])
    nb = lib.vp_batch2d_table_bytes(3)
    assert nb > 3 * 4 * 100
    tab = ctypes.create_string_buffer(nb)
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, None, tab, nb) == 0, lib.vp_last_error()
    assert tab.raw[:8] == b"VPBATCH1"
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, None, tab, nb - 1) == 3
    assert lib.vp_batch2d_plan(L.VP_F32, 0, 1, runs, 3, None, tab, nb) == 5  # diagnostics need the field
    tiles = L.BatchTiles()
    tiles.block[0] = 64
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, ctypes.byref(tiles), tab, nb) == 1
    tiles.block[0], tiles.segments[1] = 128, 3
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, ctypes.byref(tiles), tab, nb) == 1
    tiles.segments[1] = 2
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, ctypes.byref(tiles), tab, nb) == 0
    runs[1].s1 = runs[1].f
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, None, tab, nb) == 1
    runs[1].s1 = runs[1].f + 0x1000000
    runs[2].workspace_bytes = 64
    assert lib.vp_batch2d_plan(L.VP_F32, 1, 1, runs, 3, None, tab, nb) == 3
    bad = ctypes.create_string_buffer(nb)
    assert lib.vp_batch2d_step(bad, bad, 0, None, None) == 1 and b"not a batch table" in lib.vp_last_error()


def test_workspace_queries(lib):
    assert lib.vp_poisson2d_workspace_bytes(128, 128) >= 4 * 128 * 65 * 16
    assert lib.vp_drift_rho_workspace_bytes(128, 128, 128 * 128) >= 128 * 128 * 64 * 8
    assert lib.vp_step1d_workspace_bytes(4096, 4096) > 0
