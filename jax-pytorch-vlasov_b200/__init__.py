"""B200-native (sm_100a) Vlasov-Poisson step, a drop-in for the PyTorch
solvers of yasahi-hpc/JAX-PyTorch-Vlasov.

Modules:
  vlasov2d2v  -- the 2D2V API (Grid, advect_*, compute_rho, compute_poisson_real,
                 vlasov_step_*, Vlasov), same names and signatures as the reference
  vlasov1d1v  -- the 1D1V API
  engine      -- Stepper2D / Stepper1D: one library call per Strang step, CUDA graphs;
                 BatchStepper2D: many uneven runs, one launch per substep for all
  workloads   -- seeded initial conditions and the batched-runs parameter draws
  rates       -- damping and growth rates from a field-energy history
  autotune    -- tile shapes of the batched sweeps, measured and cached in JSON
  corrector   -- learned correction of the velocity-kick interpolation weights on
                 tcgen05 tensor cores: network, training on coarse / refined
                 pairs, LearnedStepper2D
  ops         -- tensor-level wrappers of the C ABI (include/vlasov_b200.h)
  build       -- compiles csrc/*.cu into libvlasov_b200.so for sm_100a

The package directory name is not a Python identifier; import it with
importlib.import_module("jax-pytorch-vlasov_b200").
"""
from . import _lib, build, ops  # noqa: F401
from ._lib import DIAG_NAMES, VlasovError, load  # noqa: F401
from .engine import BatchStepper2D, Stepper1D, Stepper2D  # noqa: F401

__all__ = ["BatchStepper2D", "Stepper1D", "Stepper2D", "VlasovError", "load", "ops", "build", "DIAG_NAMES", "vlasov2d2v",
           "vlasov1d1v"]


def __getattr__(name):
    if name in ("vlasov2d2v", "vlasov1d1v", "snapshot", "workloads", "autotune", "corrector", "slab", "rates"):
        import importlib

        return importlib.import_module(f"{__name__}.{name}")
    raise AttributeError(name)
