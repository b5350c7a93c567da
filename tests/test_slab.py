"""x-slab decomposition of one 2D2V run: the plan (host logic) and a
world-size-2 gloo run on CPU whose ranks step their slabs with the oracle's
sweeps, exchanging halo rows and gathering rho through the same calls the
GPU ranks use; the gathered result equals the whole-domain oracle step."""
import importlib
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import PACKAGE
from oracle import core as O

slab = importlib.import_module(PACKAGE + ".slab")


def test_drift_reach():
    # window rows x - s - 3 .. x - s + 2
    assert slab.drift_reach(np.array([0])) == (3, 2)
    assert slab.drift_reach(np.array([-4, 2, 5])) == (8, 6)
    assert slab.drift_reach(np.array([-9])) == (0, 11)


def test_plan_rows_and_halos():
    p = slab.SlabPlan.build(50, 3, np.array([-2, 1]))
    assert (p.hl, p.hr) == (8, 8)
    assert p.starts == (0, 16, 33, 50)
    assert [p.local(r) for r in range(3)] == [16, 17, 17]
    assert p.extended(1) == 17 + 16
    rows = p.global_rows(0)
    assert rows[0] == (0 - 8) % 50 and rows[8] == 0 and rows[-1] == (16 + 8 - 1) % 50
    # slabs thinner than the halo would need rows of a rank's neighbours'
    # neighbours: refused
    with pytest.raises(ValueError):
        slab.SlabPlan.build(20, 3, np.array([-2, 1]))
    with pytest.raises(ValueError):
        slab.SlabPlan.build(2, 3, np.array([0]))


def test_plan_sources():
    p = slab.SlabPlan.build(40, 4, np.array([0, 1]))
    assert (p.hl, p.hr) == (8, 4)
    src = p.halo_sources(0)
    assert src[0] == (3, p.local(3) - 8, 8, 0)      # the last 8 rows of rank 3
    assert src[1] == (1, 0, 4, 8 + p.local(0))      # the first 4 rows of rank 1
    # the sources are exactly the global rows of the halo
    for r in range(4):
        rows = p.global_rows(r)
        for s, first, n, dst in p.halo_sources(r):
            x0, _ = p.rows(s)
            assert list(rows[dst:dst + n]) == list(range(x0 + first, x0 + first + n))


def test_single_rank_plan():
    p = slab.SlabPlan.build(8, 1, np.array([-3, 3]))
    assert p.extended(0) == 8 + p.hl + p.hr
    f = torch.arange(p.extended(0) * 2, dtype=torch.float64).reshape(-1, 2)
    slab.exchange_halos(f, p, 0)
    rows = p.global_rows(0)
    body = f[p.hl:p.hl + 8].clone()
    for i, g in enumerate(rows):
        assert torch.equal(f[i], body[g])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


SHAPE = (24, 8, 10, 12)
LX, LY, VX, VY, DT = 4 * math.pi, 4 * math.pi, 6.0, 5.0, 0.2


def _oracle_setup():
    g = O.make_grid2d(*SHAPE, LX, LY, VX, VY, dtype=np.float64)
    st = O.Stepper2D(g, DT, window=-1)
    return g, st


def _slab_worker(rank, world, port, out_dir, steps):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, st = _oracle_setup()
        plan = slab.SlabPlan.build(g.Nx, world, st.sx)
        f = O.landau_2d(g, 0.3, 0.5)
        fe = np.ascontiguousarray(f[plan.global_rows(rank)])
        hl, n = plan.hl, plan.local(rank)
        for _ in range(steps):
            t = torch.from_numpy(fe)
            slab.exchange_halos(t, plan, rank)  # fills fe in place
            a = st.drift_y(st.drift_x(fe))
            rho = O.compute_rho(a, g.dvx, g.dvy)[hl:hl + n]
            rho_g = slab.gather_rho(torch.from_numpy(np.ascontiguousarray(rho)), plan).numpy()
            Ex, Ey, _, _ = O.compute_poisson_real(rho_g, g.kx, g.ky, g.inv_ksq)
            rows = plan.global_rows(rank)
            b = O.kick_static(a, Ex[rows], DT, g.dvx, axis=2, window=-1)
            b = O.kick_static(b, Ey[rows], DT, g.dvy, axis=3, window=-1)
            fe = np.ascontiguousarray(st.drift_x(st.drift_y(b)))
        np.save(os.path.join(out_dir, f"slab{rank}.npy"), fe[hl:hl + n])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ranks_equal_whole_domain(tmp_path, world):
    steps = 3
    mp.start_processes(_slab_worker, args=(world, _free_port(), str(tmp_path), steps), nprocs=world,
                       start_method="spawn")
    g, st = _oracle_setup()
    f = O.landau_2d(g, 0.3, 0.5)
    for _ in range(steps):
        f = st.step(f).f
    got = np.concatenate([np.load(tmp_path / f"slab{r}.npy") for r in range(world)])
    np.testing.assert_array_equal(got, f)
