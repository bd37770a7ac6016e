# cython:language_level=3
# STEPS Python binding of the drop-in solver: the module a STEPS build adds beside
# cysteps_mpi.pyx.  Like that module it includes the common bindings (cysteps.pyx: model,
# geometry, RNG and the solver API classes) and adds one solver class,
# _py_TetOpSplitB200, with _py_TetOpSplitP's constructor and solver-level methods
# (pysteps/cysteps_mpi.pyx:74-700: information, control, checkpoints, temperature, EField
# step, batch counts); the species, compartment, patch, tet, triangle and vertex accessors
# come from _py_TetAPI, and every call reaches the GPU through the C++ class.
include "cysteps.pyx"

from steps_b200 cimport TetOpSplitB200

# ----------------------------------------------------------------------------------------------------------------------
cdef class _py_TetOpSplitB200(_py_TetAPI):
    """Bindings for the GPU operator-split solver TetOpSplitB200"""
# ----------------------------------------------------------------------------------------------------------------------
    cdef TetOpSplitB200 *ptrx(self):
        return <TetOpSplitB200*> self._ptr

    def __init__(self, _py_Model model, _py_Geom geom, _py_RNG rng, int calcMembPot=0,
                 std.vector[int] tet_hosts=[], dict tri_hosts={}, std.vector[int] wm_hosts=[]):
        """
        Construction::

            sim = steps.solver.TetOpSplitB200(model, geom, rng, calcMembPot=0)

        The operator-split spatial SSA of TetOpSplit on one GPU.  The arguments are those of
        TetOpSplitP; the host lists are accepted and ignored (the whole mesh lives on one
        GPU).  calcMembPot selects the membrane-potential solver (0: none).
        """
        cdef std.map[steps.triangle_global_id, int] _tri_hosts
        for key, elem in tri_hosts.items():
            _tri_hosts[steps.triangle_global_id(key)] = elem
        if model == None:
            raise TypeError('The Model object is empty.')
        if geom == None:
            raise TypeError('The Geom object is empty.')
        if rng == None:
            raise TypeError('The RNG object is empty.')
        self._ptr = new TetOpSplitB200(model.ptr(), geom.ptr(), rng.ptr(), calcMembPot, tet_hosts, _tri_hosts,
                                       wm_hosts)


    def getSolverName(self):
        """Return a string of the solver's name."""
        return self.ptrx().getSolverName()

    def getSolverDesc(self):
        """Return a string of the solver's description."""
        return self.ptrx().getSolverDesc()

    def getSolverAuthors(self):
        """Return a string of the solver's authors."""
        return self.ptrx().getSolverAuthors()

    def getSolverEmail(self):
        """Return a string of the solver's email."""
        return self.ptrx().getSolverEmail()

    def reset(self):
        """Reset the simulation state and time to the initial values."""
        self.ptrx().reset()

    def run(self, double endtime):
        """Advance the simulation until endtime (s), at or after the current time."""
        self.ptrx().run(endtime)

    def advance(self, double adv):
        """Advance the simulation by adv seconds."""
        self.ptrx().advance(adv)

    def step(self):
        """Not available in an operator-split solver (raises, as TetOpSplitP)."""
        self.ptrx().step()

    def checkpoint(self, str file_name):
        """Write the whole simulation state to file_name."""
        self.ptrx().checkpoint(to_std_string(file_name))

    def restore(self, str file_name):
        """Load a state that checkpoint() wrote on the same model and mesh."""
        self.ptrx().restore(to_std_string(file_name))

    def setEfieldDT(self, double efdt):
        """Set the EField time step (s)."""
        self.ptrx().setEfieldDT(efdt)

    def getEfieldDT(self):
        """Return the EField time step (s)."""
        return self.ptrx().getEfieldDT()

    def setTemp(self, double t):
        """Set the temperature (K) of the GHK currents."""
        self.ptrx().setTemp(t)

    def getTemp(self):
        """Return the temperature (K)."""
        return self.ptrx().getTemp()

    def getTime(self):
        """Return the simulation time (s)."""
        return self.ptrx().getTime()

    def getNSteps(self):
        """Return the number of split windows run since the last reset."""
        return self.ptrx().getNSteps()

    def getBatchTetSpecCountsNP(self, index_t[:] index_array, str s, double[:] counts):
        """Counts of species s in the tets of index_array, into counts (gathered on the GPU)."""
        self.ptrx().getBatchTetSpecCountsNP(&index_array[0], index_array.shape[0], to_std_string(s), &counts[0],
                                            counts.shape[0])
