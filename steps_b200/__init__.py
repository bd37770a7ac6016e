"""steps_b200 — B200-native operator-split spatial SSA behind STEPS' solver API.

Submodules: ``model`` / ``geom`` / ``rng`` (inputs, reference naming), ``solver``
(TetOpSplit mirror over the C ABI of libsteps_b200.so), ``workloads`` (synthetic
Kuhn-cube configurations), ``build`` (nvcc recipe).
"""
__version__ = "0.1.0"
