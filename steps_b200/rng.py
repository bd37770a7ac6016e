"""RNG handle passed to the solver, as in the reference's ``steps.rng.create``
(src/steps/rng/create.cpp:44-56).  The solver only reads the seed: it keys
counter-based Philox4x32-10 streams, one per (realization, tet, window), instead of
consuming one buffered serial stream (src/steps/rng/r123.cpp:43-82)."""


class RNG:
    def __init__(self, name, bufsize):
        if name not in ("r123", "mt19937"):
            raise ValueError(f"unknown RNG '{name}'")
        self.name = name
        self.bufsize = int(bufsize)
        self.seed = 0

    def initialize(self, seed):
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF


def create(name, bufsize):
    return RNG(name, bufsize)
