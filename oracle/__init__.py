"""CPU oracle of the Vlasov-Poisson step: TEST INFRASTRUCTURE ONLY.

A restatement of the reference solver's algorithm (yasahi-hpc/JAX-PyTorch-Vlasov,
simulations/vlasov2d_2v/pytorch/src/vlasov2D2V.py and
simulations/vlasov1d_1v/pytorch/src/vlasov1D1V.py) in C + OpenMP and numpy,
pinned against outputs of the reference itself (tests/golden/). Only the tests,
__graft_entry__.smoke() and bench.py's CPU baseline use it, as the checker and
as the timed CPU reference; the CUDA library never calls it.
"""
